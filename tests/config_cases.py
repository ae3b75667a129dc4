"""The benchmark configurations as single-class-step test cases.

A case is the finest size class of a root run over an (nx, ny, nz) domain at
dx = dy = dz = 100 m (turbulon size k = 200 m, spheroscale 1 km, alpha = 1.8,
C1 = 0.1, H = 1/3, Hz = 5/9, seed 0; the class key is the finest of
``SeedSequence(0).spawn(n_classes)``), with a seeded synthetic state standing
in for the previous classes (no dataset exists):

* C0: 128 x 128 x 64 (the reference's own CPU-runnable configuration);
* C1: 512 x 512 x 256;
* C2: 2048 x 2048 x 256 (the headline workload).

``build(sim, shape)`` takes the module that provides the host-side set-up
functions (``_compute_all_grids``, ``_k_z``, ``_compute_normalization``,
``_bound_buffers``): the reference's ``steam.simulate`` when the golden
fixtures are generated, this package's ``steam_b200.simulate`` in the tests.
The two agree bit for bit (``tests/test_host.py`` pins the grid ladder and
the normalisation to the reference's fixtures).
"""

from __future__ import annotations

import numpy as np

ALPHA, C1, H, HZ = 1.8, 0.1, 1.0 / 3.0, 5.0 / 9.0
BOUNDS = (315 * 1004, 355 * 1004, 0.0, 0.03)
K_FINEST = 200.0
SURFACE_PRESSURE = 101325.0

C0 = (128, 128, 64)
C1_SHAPE = (512, 512, 256)
C2 = (2048, 2048, 256)


def build(sim, shape, s=1):
    """The finest class's set-up over ``shape`` at sparsity ``s`` in every
    axis (grid spacing k / (2 s): 100 m at s = 1; the 61^3 kernel at s = 5)."""
    nx, ny, nz = shape
    d = K_FINEST / (2 * s)
    height = nz * d
    zp = np.arange(int(height / (d / 2)) + 1) * (d / 2)
    hp = (340e3 - 20e3 * zp / zp[-1]).astype(np.float32)
    qp = (0.018 - 0.016 * zp / zp[-1]).astype(np.float32)
    sph = np.full(zp.size, 1000.0)
    outer = nx * d
    kv = np.array([K_FINEST])
    grids = sim._compute_all_grids(kv, nx * d, ny * d, height, (s, s, s), sph, zp)
    got = (int(grids['nx'][0]), int(grids['ny'][0]), int(grids['nz'][0]))
    assert got == tuple(shape), got
    kzl = sim._k_z('piecewise_isotropic_below_spheroscale', outer, sph)
    C_h = sim._compute_normalization(hp, zp, kzl, kv, outer, grids, hurst_horizontal=H)
    C_q = sim._compute_normalization(qp, zp, kzl, kv, outer, grids, hurst_horizontal=H)
    b_h = sim._bound_buffers(C_h, 1, H)
    b_q = sim._bound_buffers(C_q, 1, H)
    z = grids['z_arrays'][0]
    aspect = (sim._k_z('piecewise_isotropic_below_spheroscale', K_FINEST,
                       np.interp(z, zp, sph)) / K_FINEST).astype(np.float32)
    n_classes = max(1, int(round(np.log(outer / K_FINEST) / np.log(2.0))) + 1)
    seed = np.random.SeedSequence(0).spawn(n_classes)[-1]
    return dict(grids=grids, zp=zp, hp=hp, qp=qp, C_h=C_h, C_q=C_q, b_h=b_h, b_q=b_q,
                aspect=aspect, seed=seed, z=z, shape=tuple(shape), s=s, dx=d,
                h_mean=np.interp(z, zp, hp).astype(np.float32),
                qt_mean=np.interp(z, zp, qp).astype(np.float32))


def inputs(shape, seed=2026):
    """The seeded synthetic entering state (float32): h', qt', flux."""
    rng = np.random.default_rng(seed)
    h = (600.0 * rng.standard_normal(shape)).astype(np.float32)
    q = (0.0006 * rng.standard_normal(shape)).astype(np.float32)
    F = (1.0 + 0.1 * rng.random(shape)).astype(np.float32)
    return h, q, F


def sample_index(n_cells, count=16384, seed=7):
    """Sorted flat indices of the cells the golden fixture keeps."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n_cells, size=min(count, n_cells), replace=False))


def level_stats(field):
    """Per-level mean and root-mean-square (float64) of an (nx, ny, nz) field."""
    f = np.asarray(field, dtype=np.float64)
    return np.stack([f.mean(axis=(0, 1)), np.sqrt((f * f).mean(axis=(0, 1)))])


def oracle_step(O, case, h, q, F, turbulon_shape='mexican_hat', dtype=np.float64):
    """The oracle's class step and condensate map on copies of (h, q, F) in
    ``dtype``; returns (fields, record)."""
    t = np.dtype(dtype)
    h, q, F = (np.array(a, dtype=t) for a in (h, q, F))
    s = case['s']
    kern = O.turbulon_envelope(1, 0.5 / s, 0.5 / s, 0.5 / s, shape=turbulon_shape, dtype=t)
    rec, _ = O.class_step(
        h, q, F, O.class_key(case['seed']), kern, h_mean=case['h_mean'],
        qt_mean=case['qt_mean'], z_coords=case['z'], dx=case['dx'], dy=case['dx'],
        aspect=case['aspect'], C_h=case['C_h'][0], C_qt=case['C_q'][0], b_h=case['b_h'][0],
        b_qt=case['b_q'][0], h_min=BOUNDS[0], h_max=BOUNDS[1], qt_min=BOUNDS[2],
        qt_max=BOUNDS[3], flux_noise_scale=C1, n_per_dyad=1, sparsity_factors=(s, s, s),
        n_zero=2 * s, alpha=ALPHA)
    hm = case['h_mean'].astype(t)
    qm = case['qt_mean'].astype(t)
    diag = O.recover_diagnostics(np.clip(h + hm, BOUNDS[0], BOUNDS[1]),
                                 np.clip(q + qm, BOUNDS[2], BOUNDS[3]), case['z'],
                                 SURFACE_PRESSURE)
    fields = {"flux": F, "h": h, "qt": q, "qc": diag['qc'], "qi": diag['qi'], "T": diag['T']}
    return fields, rec


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def log_flux_error(F, F_ref, clip_band=1e-3):
    """log-flux relative L2 over the cells where both fields are clear of the
    clip (F > clip_band), with the rest reported apart: the count of cells
    whose clip state differs, and the largest absolute flux difference among
    cells within the clip band (where F + T * (eps F) nearly cancels and log F
    of an O(1e-6) value carries no relative precision)."""
    F = np.asarray(F, dtype=np.float64)
    F_ref = np.asarray(F_ref, dtype=np.float64)
    clear = (F_ref > clip_band) & (F > clip_band)
    both_clipped = (F_ref == 0) & (F == 0)
    near = ~clear & ~both_clipped
    return {"log_flux_rel_l2": rel_l2(np.log(F[clear]), np.log(F_ref[clear])),
            "clip_mask_differs": int(np.count_nonzero((F > 0) != (F_ref > 0))),
            "near_clip_cells": int(np.count_nonzero(near)),
            "near_clip_max_abs": float(np.max(np.abs(F[near] - F_ref[near]))) if near.any()
            else 0.0}


def device_step(sim, thermo, case, h, q, F, dtype, turbulon_shape='mexican_hat',
                resident=False):
    """The CUDA path's class step through its ``cascade_loop`` (the call the
    reference makes, steam/simulate.py:1566) and the condensate map; returns
    the fields as numpy arrays, or as CUDA tensors with ``resident``."""
    s = case['s']
    out = sim.cascade_loop(
        case['hp'], case['qp'], case['zp'], case['grids'], case['C_h'], case['C_q'],
        case['b_h'], case['b_q'], [case['aspect']], *BOUNDS, 1, (s, s, s), [case['seed']],
        h_perturbation=h, qt_perturbation=q, flux=F, flux_noise_scale=C1,
        turbulon_shape=turbulon_shape, comp_k=[np.ones(case['shape'][2], np.float32)],
        dtype=dtype, resident=True)
    h_o, q_o, F_o = out[0], out[1], out[2]
    diag = thermo.recover_diagnostics_device(
        h_o, q_o, case['z'], SURFACE_PRESSURE, h_mean=case['h_mean'],
        qt_mean=case['qt_mean'], bounds=np.asarray(BOUNDS, np.float64))
    fields = {"flux": F_o, "h": h_o, "qt": q_o, "qc": diag['qc'], "qi": diag['qi'],
              "T": diag['T']}
    if not resident:
        fields = {k: v.cpu().numpy() for k, v in fields.items()}
    return fields, out[7].classes[0]
