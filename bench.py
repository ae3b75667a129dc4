#!/usr/bin/env python
"""Throughput of the STEAM field step on B200: Mvoxels/s at 2048^2 x 256 FP32.

Workload: the finest size class of the 2048 x 2048 x 256 domain (dx = dz =
100 m, k = 200 m; alpha = 1.8, C1 = 0.1, H = 1/3, Hz = 5/9, spheroscale 1 km,
seed 0) taken through one cascade class -- world-keyed Philox noise, extremal
Levy multiplier, flux convolution with clip and unit-mean restore, advective
weight x signed amplitude x bound taper for h and qt, second convolution,
bounded amplitude-preserving add -- and the thermodynamic map to condensate.
Synthetic seeded state (flux, h', qt') with those shapes stands in for the
previous classes; there is no dataset.  Every field (4.3 GB) is larger than
L2, so no flush is needed between steps.

`value`: device-resident, CUDA events on the launching stream, max over
ranks.  `e2e`: the same step through the public host-array API
(steam_b200.simulate.field_step) with pinned host inputs/outputs, transfers
inside the timed region.  `--impl reference` times the CPU oracle port of the
same step on a bounded sub-box on the host cores.

Launch: python bench.py [--gpus N --steps K --warmup W]; for N > 1 under
torchrun, each rank advances its own independent field (replicas).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

METRIC = "Mvoxels/s at 2048^2x256 FP32 (field step: noise, flux, 2 scalar convolutions, bounded add, condensate)"
ALPHA, C1, H, HZ = 1.8, 0.1, 1.0 / 3.0, 5.0 / 9.0
BOUNDS = (315 * 1004, 355 * 1004, 0.0, 0.03)
# Algorithmic HBM bytes per voxel of one FP32 field step: flux read+write (8),
# h' and qt' read+write (16), qc and qi written (8).
STEP_BYTES_PER_VOXEL = 32


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=2048)
    ap.add_argument("--nz", type=int, default=256)
    ap.add_argument("--dtype", choices=("f32", "f64"), default="f32")
    ap.add_argument("--shape", choices=("mexican_hat", "morlet_omega0_6"),
                    default="mexican_hat",
                    help="turbulon shape: the Mexican hat factors into separable "
                         "filters; the Morlet runs the FFT convolution")
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--cpu-sample", type=int, nargs=3, default=(128, 128, 256),
                    metavar=("NX", "NY", "NZ"))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-error", action="store_true",
                    help="skip the float64 step that states the benched step's error")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="tile requests per arrival rate in the serving episode, at most "
                         "2 s of arrivals and at least 20 (0: skip)")
    ap.add_argument("--serve-rates", type=float, nargs="+",
                    default=(10.0, 100.0, 1000.0, 2000.0),
                    help="Poisson arrival rates (requests/s) of the serving episode")
    ap.add_argument("--ensemble-members", type=int, default=256,
                    help="members of the batched-ensemble episode (0: skip)")
    ap.add_argument("--no-k61", dest="k61", action="store_false",
                    help="skip the 61^3-kernel convolution at 512x512x256")
    ap.add_argument("--streamed-steps", type=int, default=1,
                    help="out-of-core class steps of the workload with its fields in "
                         "page-locked host memory (0: skip)")
    ap.add_argument("--streamed-tile", type=int, default=512,
                    help="column tile of the out-of-core step (plus a 7-cell halo)")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# Workload setup (host, shared by both arms)
# ---------------------------------------------------------------------------

def config_dict(shape, world, turbulon_shape="mexican_hat"):
    """The workload's config, the same for both arms."""
    return {"workload": f"field step at {shape[0]}x{shape[1]}x{shape[2]} "
                        f"(finest class of the {shape[0]}x{shape[1]}x{shape[2]} domain, "
                        f"k=200 m, dx=dz=100 m) + condensate",
            "turbulon": turbulon_shape,
            "alpha": ALPHA, "C1": C1, "H": H, "Hz": HZ, "seed": 0,
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (4.3 GB fields); no flush"}


def workload(nx, ny, nz):
    from steam_b200 import simulate as sim
    height = nz * 100.0
    zp = np.arange(int(height / 50.0) + 1) * 50.0
    hp = (340e3 - 20e3 * zp / zp[-1]).astype(np.float32)
    qp = (0.018 - 0.016 * zp / zp[-1]).astype(np.float32)
    sph = np.full(zp.size, 1000.0)
    k = 200.0
    outer = nx * 100.0
    grids = sim._compute_all_grids(np.array([k]), nx * 100.0, ny * 100.0, height, (1, 1, 1),
                                   sph, zp)
    shape = (int(grids['nx'][0]), int(grids['ny'][0]), int(grids['nz'][0]))
    assert shape == (nx, ny, nz), shape
    kzl = sim._k_z('piecewise_isotropic_below_spheroscale', outer, sph)
    C_h = sim._compute_normalization(hp, zp, kzl, np.array([k]), outer, grids,
                                     hurst_horizontal=H)[0]
    C_q = sim._compute_normalization(qp, zp, kzl, np.array([k]), outer, grids,
                                     hurst_horizontal=H)[0]
    b_h = sim._bound_buffers([C_h], 1, H)[0]
    b_q = sim._bound_buffers([C_q], 1, H)[0]
    aspect = (sim._k_z('piecewise_isotropic_below_spheroscale', k,
                       np.interp(grids['z_arrays'][0], zp, sph)) / k).astype(np.float32)
    # finest class key of a seed-0 root run over this domain
    n_classes = int(round(np.log(outer / 200.0) / np.log(2.0))) + 1
    key = sim.class_key(np.random.SeedSequence(0).spawn(n_classes)[-1])
    return dict(sim=sim, grids=grids, zp=zp, hp=hp, qp=qp, C_h=C_h, C_q=C_q, b_h=b_h,
                b_q=b_q, aspect=aspect, key=key, shape=shape)


# ---------------------------------------------------------------------------
# Clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    """SM clocks and clock-event reasons sampled every 200 ms during the timed
    region, from NVML in a thread of this process.  (A polling nvidia-smi
    process stalls this process's CUDA calls while it queries: the field step
    ran at half speed under it.)"""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, gpu_index, period=0.2):
        self.gpu = gpu_index
        self.period = period
        self.rows = []
        self.thread = None

    def _handle(self, nv):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            return nv.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = self._handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
        except Exception:
            self.thread = None
            return
        self.stop_ev = threading.Event()

        def run():
            while not self.stop_ev.is_set():
                try:
                    sm = self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)
                    rs = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    self.rows.append((sm, rs))
                except Exception:
                    pass
                self.stop_ev.wait(self.period)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        self.stop_ev.set()
        self.thread.join()
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"],
                    "samples": 0}
        sm = [float(r[0]) for r in self.rows]
        reasons = sorted({name for _, bits in self.rows for name, bit in self.REASONS
                          if bits & bit})
        loaded = [v for v in sm if v > 0.5 * self.max_mhz] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": float(self.max_mhz),
                "reasons": reasons, "samples": len(self.rows), "source": "nvml"}


# ---------------------------------------------------------------------------
# Per-call device timing (one instrumented step, outside the timed region)
# ---------------------------------------------------------------------------

class CallTimer:
    """Wraps the library's entry points with CUDA events on torch's current
    stream (the stream every call is launched on)."""

    def __init__(self, lib, torch):
        self.lib, self.torch = lib, torch
        self.records = []
        self.saved = {}

    def __enter__(self):
        from steam_b200 import _lib
        for name in _lib.exported_symbols():
            fn = getattr(self.lib, name)
            self.saved[name] = fn

            def wrapped(*args, _fn=fn, _name=name):
                s = self.torch.cuda.Event(enable_timing=True)
                e = self.torch.cuda.Event(enable_timing=True)
                s.record()
                rc = _fn(*args)
                e.record()
                self.records.append((_name, s, e))
                return rc
            setattr(self.lib, name, wrapped)
        return self

    def __exit__(self, *exc):
        for name, fn in self.saved.items():
            setattr(self.lib, name, fn)

    def totals(self):
        self.torch.cuda.synchronize()
        out = {}
        for name, s, e in self.records:
            if name.endswith("workspace_bytes") or name in ("steam_last_error",
                                                           "steam_launch_count"):
                continue
            t, n = out.get(name, (0.0, 0))
            out[name] = (t + s.elapsed_time(e), n + 1)
        return out


# ---------------------------------------------------------------------------
# CPU baseline: the oracle port of the same step on a bounded sub-box
# ---------------------------------------------------------------------------

def cpu_step(nx, ny, nz):
    """Time one oracle field step on (nx, ny, nz); returns (seconds, threads)."""
    from oracle import steam_oracle as O
    w = workload(nx, ny, nz)
    z = w['grids']['z_arrays'][0]
    hm = np.interp(z, w['zp'], w['hp']).astype(np.float32)
    qm = np.interp(z, w['zp'], w['qp']).astype(np.float32)
    rng = np.random.default_rng(1)
    shape = (nx, ny, nz)
    h = (600.0 * rng.standard_normal(shape)).astype(np.float32)
    q = (0.0006 * rng.standard_normal(shape)).astype(np.float32)
    F = (1.0 + 0.1 * rng.random(shape)).astype(np.float32)
    kern = O.turbulon_envelope(1, 0.5, 0.5, 0.5)
    t0 = time.perf_counter()
    O.class_step(h, q, F, tuple(int(k) for k in w['key']), kern, h_mean=hm, qt_mean=qm,
                 z_coords=z, dx=100.0, dy=100.0, aspect=w['aspect'], C_h=w['C_h'],
                 C_qt=w['C_q'], b_h=w['b_h'], b_qt=w['b_q'], h_min=BOUNDS[0],
                 h_max=BOUNDS[1], qt_min=BOUNDS[2], qt_max=BOUNDS[3], flux_noise_scale=C1,
                 n_per_dyad=1, sparsity_factors=(1, 1, 1), n_zero=2, alpha=ALPHA)
    O.recover_diagnostics(np.clip(h + hm, BOUNDS[0], BOUNDS[1]),
                          np.clip(q + qm, BOUNDS[2], BOUNDS[3]), z, 101325.0)
    return time.perf_counter() - t0, O.N_THREADS


def cpu_baseline(sample):
    nx, ny, nz = sample
    secs, threads = cpu_step(nx, ny, nz)
    return {"value": nx * ny * nz / secs / 1e6, "unit": "Mvoxels/s", "cores": threads,
            "kind": "port",
            "sample": f"one oracle field step on a {nx}x{ny}x{nz} sub-box of the workload "
                      f"({secs:.1f} s on {threads} host threads; numpy/scipy restatement "
                      f"of the reference's CPU path)"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    nx, ny, nz = args.cpu_sample
    for _ in range(max(0, args.warmup) and 1):
        cpu_step(min(nx, 32), min(ny, 32), nz)
    times = []
    threads = 1
    for _ in range(max(1, args.steps)):
        secs, threads = cpu_step(nx, ny, nz)
        times.append(secs)
    per = float(np.mean(times))
    value = nx * ny * nz / per / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": "Mvoxels/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.dtype.replace("f", "f"), "data": "synthetic (seeded)",
        "impl": "reference",
        "config": config_dict((args.nx, args.ny, args.nz), world, args.shape),
        "cpu_baseline": {"value": value, "unit": "Mvoxels/s", "cores": threads,
                         "kind": "port",
                         "sample": f"the oracle's class step + condensate on a {nx}x{ny}x{nz} "
                                   f"sub-box of the workload per step, mean of {len(times)} "
                                   f"steps on {threads} host threads; the reference is Python "
                                   f"and its source does not travel to the GPU host, so its "
                                   f"CPU path is timed through this restatement, which the "
                                   f"tests pin to the reference's own run at 128x128x64"},
        "e2e": {"value": value, "unit": "Mvoxels/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Error of the benched float32 step against float64
# ---------------------------------------------------------------------------

def float64_error(torch, sim, w, h0, q0, F0, F, hp, qp, diag, turbulon_shape, clip_band=1e-3):
    """Run the same class step in float64 on the device from the same inputs
    and return the float32 result's error against it: log-flux relative L2
    over the cells clear of the clip (F > clip_band in both), the count of
    cells whose clip state differs, the largest absolute flux difference on
    the cells within the clip band, and relative L2 of the h and qt
    increments and of qc and qi."""
    from steam_b200 import resident as _resident
    setup64 = sim.make_class_setup(
        w['grids'], 0, h_profile=w['hp'], qt_profile=w['qp'], z_profile=w['zp'],
        C_h=w['C_h'], C_qt=w['C_q'], b_h=w['b_h'], b_qt=w['b_q'], aspect=w['aspect'],
        bounds=BOUNDS, key=w['key'], flux_noise_scale=C1, flux_alpha=ALPHA,
        turbulon_shape=turbulon_shape, dtype=np.float64)
    h64, q64, F64 = h0.double(), q0.double(), F0.double()
    d64 = {k: torch.empty_like(h64) for k in ("T", "qv", "qc", "qi", "p")}
    r64 = _resident.ResidentClass(setup64, torch.float64)
    r64.step(h64, q64, F64, diagnostics=d64)
    torch.cuda.synchronize()
    r64.work = None
    del r64, d64["T"], d64["qv"], d64["p"]
    torch.cuda.empty_cache()

    def rel(a, b):
        return float(torch.linalg.vector_norm((a.double() - b).double())
                     / torch.linalg.vector_norm(b.double()))

    Fd = F.double()
    clear = (F64 > clip_band) & (Fd > clip_band)
    both = (F64 == 0) & (Fd == 0)
    near = ~clear & ~both
    lr = torch.log(F64[clear])
    out = {"log_flux_rel_l2": float(torch.linalg.vector_norm(torch.log(Fd[clear]) - lr)
                                    / torch.linalg.vector_norm(lr)),
           "clip_mask_differs": int(((Fd > 0) != (F64 > 0)).sum()),
           "near_clip_cells": int(near.sum()),
           "near_clip_max_abs": float((Fd[near] - F64[near]).abs().max())
           if bool(near.any()) else 0.0,
           # the tests' bar on those cells: 8 float32 ulps of the entering flux
           "near_clip_bar": 8 * float(np.finfo(np.float32).eps) * float(F0.abs().max()),
           "cells": int(F.numel())}
    del Fd, clear, both, near, lr, F64
    out["h_increment_rel_l2"] = rel(hp.double() - h0.double(), h64 - h0.double())
    del h64
    out["qt_increment_rel_l2"] = rel(qp.double() - q0.double(), q64 - q0.double())
    del q64
    out["qc_rel_l2"] = rel(diag["qc"], d64["qc"])
    out["qi_rel_l2"] = rel(diag["qi"], d64["qi"])
    out["against"] = ("the same class step in float64 on the device, same inputs "
                      "(the float64 step is held to 1e-9 of the FP64 oracle at "
                      "512x512x256 in the tests)")
    return out


# ---------------------------------------------------------------------------
# Replicas: one independent workload per rank, timed as the slowest rank
# ---------------------------------------------------------------------------

def slowest_rank_ms(ms, world, device):
    """The max over ranks of a per-rank elapsed time (every rank calls it)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_mvox(nvox, ms, world):
    """Whole-job Mvoxels/s of one workload per rank in ``ms``."""
    return world * nvox / (ms / 1e3) / 1e6


def replica_throughput(nvox, steps, ms, world):
    """Whole-job Mvoxels/s: every rank processed ``steps`` workloads of ``nvox``
    voxels; ``ms`` is the slowest rank's time."""
    return world * nvox * steps / (ms / 1e3) / 1e6


# ---------------------------------------------------------------------------
# Device arm
# ---------------------------------------------------------------------------

def main(argv=None):
    args = parse(argv)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from steam_b200 import _lib
    lib = _lib.load()
    np_t = np.float32 if args.dtype == "f32" else np.float64
    tdt = torch.float32 if args.dtype == "f32" else torch.float64
    w = workload(args.nx, args.ny, args.nz)
    sim = w['sim']
    shape = w['shape']
    nvox = shape[0] * shape[1] * shape[2]
    setup = sim.make_class_setup(
        w['grids'], 0, h_profile=w['hp'], qt_profile=w['qp'], z_profile=w['zp'],
        C_h=w['C_h'], C_qt=w['C_q'], b_h=w['b_h'], b_qt=w['b_q'], aspect=w['aspect'],
        bounds=BOUNDS, key=w['key'], flux_noise_scale=C1, flux_alpha=ALPHA,
        turbulon_shape=args.shape, dtype=np_t)
    from steam_b200.resident import resident_for

    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234 + rank)
    h0 = 600.0 * torch.randn(shape, generator=gen, device="cuda", dtype=tdt)
    q0 = 0.0006 * torch.randn(shape, generator=gen, device="cuda", dtype=tdt)
    F0 = 1.0 + 0.1 * torch.rand(shape, generator=gen, device="cuda", dtype=tdt)
    hp, qp, F = h0.clone(), q0.clone(), F0.clone()
    diag = {k: torch.empty_like(hp) for k in ("T", "qv", "qc", "qi", "p")}
    resident = resident_for(setup, tdt)

    def reset():
        # every step starts from the same input state, so each step is the
        # same class step on the same data
        hp.copy_(h0)
        qp.copy_(q0)
        F.copy_(F0)

    def step():
        # the step enqueues its work and its ledger copy without waiting on
        # the GPU
        resident.step(hp, qp, F, diagnostics=diag)

    for _ in range(max(0, args.warmup)):
        reset()
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.steam_launch_count()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    # per-entry device time for the roofline, from CUDA events recorded
    # around every library call of the timed steps (on the launching stream)
    timer = CallTimer(lib, torch)
    # the steps are timed by events recorded after each step's input reset
    # (three device copies of the fields, 3 x 2 x 4.3 GB at 2048^2x256, not
    # part of the class step) and after the step, on the launching stream; the
    # whole bracket, resets included, is reported beside it
    step_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
    with timer:
        t_start.record()
        for i in range(args.steps):
            reset()
            step_events[i][0].record()
            step()
            step_events[i][1].record()
        t_end.record()
    torch.cuda.synchronize()
    launches = lib.steam_launch_count() - launches0
    if world > 1:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in step_events)
    ms_bracket = t_start.elapsed_time(t_end)
    clk = clocks.stop()
    ms = slowest_rank_ms(ms, world, "cuda")
    ms_bracket = slowest_rank_ms(ms_bracket, world, "cuda")
    ms_per_step = ms / max(args.steps, 1)
    value = replica_throughput(nvox, args.steps, ms, world)

    cl = resident.class_ledger()
    calls = timer.totals()
    ba_sweeps = {k: int(v.n_sweeps) for k, v in cl.bounded_add.items()}
    dominant = max(calls.items(), key=lambda kv: kv[1][0])
    elem = 4 if args.dtype == "f32" else 8
    # algorithmic bytes of one launch of each entry point at this shape
    # (the convolution entry runs three times a step: the flux convolution,
    # 3 fields of traffic, and two scalar convolutions, 2 fields each)
    alg = {
        "steam_conv_separable_async": 7 * elem * nvox / 3,  # mean over the three launches
        "steam_conv_fft_async": 7 * elem * nvox / 3,        # the same three launches
        "steam_conv_direct_async": 7 * elem * nvox / 3,
        "steam_flux_noise_async": 2 * elem * nvox,          # read flux, write product
        "steam_flux_finish_async": 2 * elem * nvox,         # read and write flux
        "steam_scalar_pattern_async": 3 * elem * nvox,      # read pert + product, write W
        "steam_bounded_add_async": 3 * elem * nvox,         # read pert + increment, write pert
        "steam_thermo_async": 7 * elem * nvox,              # read h', qt'; write T, qv, qc, qi, p
    }
    name, (tot_ms, n_calls) = dominant
    per_launch_ms = tot_ms / n_calls
    peaks = {}
    try:
        peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg.get(name, 2 * elem * nvox) / (per_launch_ms / 1e3) / 1e9
    # measured DRAM traffic per launch: dram__bytes_read.sum + dram__bytes_write.sum
    # of each entry's kernels in an ncu capture at 512x512x256 FP32, per voxel;
    # the kernels stream their fields once, so the traffic scales with voxels
    # (the convolution figure is the mean of its flux launch and two scalar ones)
    # (the bounded add's figure sums its first sweep, two persistent phases and
    # apply sweep: the solve streams d and the perturbation about 5 times)
    dram_per_voxel = {"steam_conv_separable_async": 9.19, "steam_thermo_async": 29.77,
                      "steam_flux_noise_async": 7.45, "steam_scalar_pattern_async": 14.96,
                      "steam_flux_finish_async": 7.13, "steam_bounded_add_async": 32.58}
    traffic = (dram_per_voxel[name] * nvox if args.dtype == "f32" and name in dram_per_voxel
               else None)
    # the instruction-issue roofline beside it: warp instructions per voxel of
    # each entry's kernels in the same ncu capture (512x512x256 FP32;
    # smsp__inst_executed.sum / voxels; the convolution figure is the mean of
    # its flux launch and two scalar ones) against 4 warp instructions per
    # cycle per SM at the SM clock sampled during the timed region
    inst_per_voxel = {"steam_conv_separable_async": 3.617, "steam_thermo_async": 8.480,
                      "steam_flux_noise_async": 7.781, "steam_scalar_pattern_async": 2.497,
                      "steam_flux_finish_async": 0.107, "steam_bounded_add_async": 5.87}
    issue = None
    if args.dtype == "f32" and name in inst_per_voxel:
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz")
        if mhz:
            ach = inst_per_voxel[name] * nvox / (per_launch_ms / 1e3) / 1e9
            pk = sms * 4 * mhz * 1e6 / 1e9
            issue = {"achieved": ach, "peak": pk, "unit": "G warp instructions/s",
                     "frac": ach / pk, "inst_per_voxel": inst_per_voxel[name],
                     "sm_mhz": mhz, "sms": sms}
    # the autotuner's choice for the convolution at this shape (CTA tile
    # height x x chunk, timed once at set-up; 0 = the kernel's wave model)
    conv_tuning = None
    from steam_b200 import ensemble as _ens
    tuned = _ens._TUNED.get((tuple(shape), tdt))
    if tuned:
        best = min(tuned, key=tuned.get)
        conv_tuning = {"rows": int(best[0]), "chunk": int(best[1]),
                       "ms": round(tuned[best], 3),
                       "model_chunk_ms": round(tuned.get((32, 0), float("nan")), 3),
                       "candidates": len(tuned)}
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic / 1e9 if traffic is not None else None,
                "traffic_unit": "GB per launch (ncu, 512x512x256 capture scaled by voxels)",
                "per_launch_ms": per_launch_ms,
                "peak_source": "measured" if peaks else "fallback",
                # the convolutions, noise and thermodynamics issue hundreds of
                # instructions per voxel: their limiter is instruction issue
                # (ncu issue-active 55-76 %), not DRAM, hence the low fraction;
                # the bounded add's solve sweeps its fields several times
                "limiter": ("the solve's repeated sweeps (DRAM traffic about 2.7x the "
                            "algorithmic bytes) and its grid barriers"
                            if name == "steam_bounded_add_async" else
                            "instruction issue (FP32/FP64 pipes), not DRAM"),
                "issue": issue,
                "bounded_add_sweeps": ba_sweeps,
                "conv_tuning": conv_tuning,
                "breakdown_ms_per_step": {k: round(v[0] / max(args.steps, 1), 3)
                                          for k, v in sorted(calls.items(),
                                                             key=lambda kv: -kv[1][0])}}

    # the benched step's error against the same step in float64 on the same
    # inputs (the float64 device step is the one the tests pin to the FP64
    # oracle at 512x512x256): after the timed steps F, hp, qp and diag hold
    # one step from (F0, h0, q0)
    error = None
    if args.dtype == "f32" and not args.no_error:
        for k in ("T", "qv", "p"):
            diag.pop(k)
        resident.work = None
        torch.cuda.empty_cache()
        error = float64_error(torch, sim, w, h0, q0, F0, F, hp, qp, diag, args.shape)
        torch.cuda.empty_cache()

    # end to end through the public host-array API, pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        def pinned_copy(t):
            host = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            host.copy_(t)
            return host.numpy()
        h_host, q_host, F_host = pinned_copy(hp), pinned_copy(qp), pinned_copy(F)
        del diag
        out_host = {k: torch.empty(shape, dtype=tdt, pin_memory=True).numpy()
                    for k in ("qc", "qi")}
        sim.field_step(h_host, q_host, F_host, setup, out=out_host)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        # K chained steps on the same arrays: each call returns before its
        # downloads finish, the next call's uploads wait for the download of
        # the same array and overlap the rest; the last result is waited for
        # inside the timed region
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        pending = None
        for _ in range(args.e2e_steps):
            pending = sim.field_step(h_host, q_host, F_host, setup, out=out_host, wait=False)
        pending.result()
        e1.record()
        torch.cuda.synchronize()
        total = slowest_rank_ms(e0.elapsed_time(e1), world, "cuda")
        e2e = {"value": replica_throughput(nvox, args.e2e_steps, total, world),
               "unit": "Mvoxels/s", "h2d_bytes_per_step": 3 * elem * nvox,
               "d2h_bytes_per_step": 5 * elem * nvox,
               "api": "steam_b200.simulate.field_step (numpy in, numpy out; page-locked "
                      "host arrays; transfers pipelined against the step and, with "
                      "wait=False, against the neighbouring steps)"}
        del h_host, q_host, F_host, out_host

    # serving: world-coordinate cube tiles (32^3..256^3, weights .4/.3/.2/.1)
    # from one world (seed 7) under Poisson arrivals, continuous batching over
    # four CUDA streams; latency = arrival to tile on the host
    serving = None
    if args.serve_requests > 0:
        from steam_b200.serving import TileServer, TileWorld, latency_summary, poisson_trace
        tw = TileWorld((args.nx, args.ny, args.nz), seed=7, dtype=np_t)
        torch.cuda.empty_cache()
        srv = TileServer(tw, n_slots=4, max_n=min(256, args.nz))
        srv.serve(poisson_trace(tw, rate=1000.0, n_requests=16, seed=5))  # warm-up
        serving = {"world": f"{args.nx}x{args.ny}x{args.nz}, seed 7",
                   "sizes": "32^3/64^3/128^3/256^3 at 0.4/0.3/0.2/0.1",
                   "slots": 4, "budget_bytes": srv.budget}
        for rate in args.serve_rates:
            nreq = min(args.serve_requests, max(20, int(2.0 * rate)))
            done = srv.serve(poisson_trace(tw, rate, nreq, seed=4))
            serving[f"{rate:g}_req_per_s"] = latency_summary(done)
        del srv, tw

    # batched ensemble: members of uneven sizes (64^3 .. 256x256x128, log-uniform)
    # and parameters, over eight streams, eagerly and from one captured CUDA
    # graph; beside it the plain FP64 drop-in (stage by stage, float64) on the
    # same members
    ensemble = None
    if args.ensemble_members > 0:
        from steam_b200.ensemble import Ensemble, config_members, plain_fp64_throughput
        members = config_members(args.ensemble_members)
        ens = Ensemble(members, n_streams=8)
        eager = ens.throughput(steps=3, graph=False)
        ens.check()
        graph = ens.throughput(steps=3, graph=True)
        ens.check()
        ensemble = {"members": len(members), "voxels": ens.voxels,
                    "grouped_bounded_adds": ens.grouped,
                    "eager_fp32": eager, "graph_fp32": graph}
        ens.release()
        del ens, members
        torch.cuda.empty_cache()
        # the same members in float64: the resident graph (precision apart
        # from API) and the plain stage-by-stage drop-in (API apart)
        members = config_members(args.ensemble_members, dtype=np.float64)
        ens = Ensemble(members, n_streams=8, tune=False)
        ensemble["graph_fp64"] = ens.throughput(steps=2, graph=True)
        ens.check()
        ens.release()
        del ens
        torch.cuda.empty_cache()
        ensemble["plain_fp64_stagewise"] = plain_fp64_throughput(members, steps=1)
        r = {k: ensemble[k]["mvoxels_per_s"] for k in ("graph_fp32", "graph_fp64",
                                                       "plain_fp64_stagewise")}
        ensemble["graph_fp32_over_plain_fp64"] = r["graph_fp32"] / r["plain_fp64_stagewise"]
        ensemble["graph_fp64_over_plain_fp64"] = r["graph_fp64"] / r["plain_fp64_stagewise"]
        ensemble["graph_fp32_over_graph_fp64"] = r["graph_fp32"] / r["graph_fp64"]
        del members
        torch.cuda.empty_cache()

    # the 61^3 kernel (sparsity 5: the 512x512x256 configuration's
    # "64-voxel kernel support"): one float32 convolution at 512x512x256,
    # which runs as the separable z/y/x passes (a 61-tap ring does not fit
    # the fused kernels' registers)
    k61 = None
    if args.k61 and args.dtype == "f32":
        from steam_b200 import simulate as _sim
        from steam_b200 import utils as _u
        shp = (512, 512, 256)
        kern = _sim._turbulon_envelope(1, 0.1, 0.1, 0.1, dtype=np.float64)
        plan = _u.plan_convolution(kern, shp, np.float32)
        fk = torch.randn(shp, device="cuda")
        ok = torch.empty_like(fk)
        for _ in range(2):
            _u.run_plan_async(plan, fk, ok)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            _u.run_plan_async(plan, fk, ok)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 3
        k61 = {"kernel": list(kern.shape), "shape": list(shp), "plan": plan.kind,
               "ms": round(ms, 3), "mvoxels_per_s": fk.numel() / (ms / 1e3) / 1e6}
        del fk, ok
        torch.cuda.empty_cache()

    # out-of-core: the same class step with h', qt', F in page-locked host
    # memory, column tiles (+ halo) and level slabs streamed through the
    # device, transfers overlapped with compute on three streams
    streamed = None
    if args.streamed_steps > 0:
        from steam_b200.outofcore import host_scratch, streamed_class_step
        torch.cuda.empty_cache()
        scratch = host_scratch(shape, np_t)
        host = {}
        for k, t in (('h', h0), ('qt', q0), ('F', F0)):
            host[k] = torch.empty(shape, dtype=tdt, pin_memory=True)
            host[k].copy_(t)
        outs = {k: torch.empty(shape, dtype=tdt, pin_memory=True).numpy() for k in ('qc', 'qi')}
        keep = {k: v.clone() for k, v in host.items()}
        del h0, q0, F0, hp, qp, F
        torch.cuda.empty_cache()
        tile = (args.streamed_tile, args.streamed_tile)
        times = []
        for _ in range(args.streamed_steps):
            for k in host:
                host[k].copy_(keep[k])
            torch.cuda.synchronize()
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record()
            streamed_class_step(host['h'].numpy(), host['qt'].numpy(), host['F'].numpy(), setup,
                                tile=tile, slab_levels=32, out=outs, scratch=scratch)
            s1.record()
            torch.cuda.synchronize()
            times.append(s0.elapsed_time(s1))
        ms = slowest_rank_ms(min(times), world, "cuda")
        streamed = {"mvoxels_per_s": replicas_mvox(nvox, ms, world), "ms_per_step": ms,
                    "tile": list(tile), "halo": 7, "slab_levels": 32,
                    "note": "fields in page-locked host memory; per class step: flux "
                            "measure, pattern measure, two second convolutions, bounded "
                            "adds on level slabs, restore + thermodynamics"}
        del host, keep, outs, scratch

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(tuple(args.cpu_sample))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mvoxels/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "ms_per_step_with_resets": ms_bracket / max(args.steps, 1),
            "timing": "each step between CUDA events on the launching stream, recorded "
                      "after the step's input reset (3 field copies) and after the step; "
                      "ms_per_step_with_resets is the whole bracket",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.dtype, "data": "synthetic (seeded state and noise)",
            "config": config_dict(shape, world, args.shape),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "error": error,
            "streamed": streamed, "serving": serving,
            "ensemble": ensemble,
            "k61": k61,
            "gpu_launches": int(launches), "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
