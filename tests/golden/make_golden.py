"""Generate the golden fixtures by running the reference.

The reference implementation (thomasdewitt/STEAM, pure Python + numba) is
imported read-only from its source tree, whose path is the required first
argument, with two shims: a one-line ``netCDF4`` import stub (the package
imports netCDF4 at module load; nothing here writes NetCDF) and a scratch
NUMBA_CACHE_DIR so that no shipped numba cache is read.

Two files:

* ``reference_fixtures.npz``: inputs and the reference's outputs for the
  hot-path stages at toy sizes (``--part unit``);
* ``c0_class_step.npz``: the reference's own single class step at the
  128 x 128 x 64 configuration (``tests/config_cases.py``; seed 0, alpha 1.8,
  C1 0.1, H 1/3, Hz 5/9), for the Mexican-hat and the Morlet turbulon, through
  its ``cascade_loop`` on the finest class's grid and its
  ``recover_diagnostics``: the ledger scalars in full, the fields' per-level
  mean and RMS in full, and a fixed sample of 16,384 cells of every field
  (``--part c0``).

The tests compare the oracle (and, on a GPU, the CUDA path) against these
arrays; the reference itself is never needed at test time.

Run: python tests/golden/make_golden.py /path/to/reference [--part unit|c0|all]
"""

from __future__ import annotations

import importlib
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "reference_fixtures.npz"


def _import_reference(ref_root: Path):
    stub_dir = Path(tempfile.mkdtemp(prefix="steam_golden_stub_"))
    (stub_dir / "netCDF4.py").write_text(
        "class Dataset:\n"
        "    def __init__(self, *a, **k):\n"
        "        raise RuntimeError('netCDF4 is stubbed for fixture generation')\n")
    os.environ.setdefault("NUMBA_CACHE_DIR", str(Path(tempfile.mkdtemp(prefix="numba_"))))
    sys.path.insert(0, str(stub_dir))
    sys.path.insert(0, str(ref_root))
    sim = importlib.import_module("steam.simulate")
    noise = importlib.import_module("steam.noise")
    utils = importlib.import_module("steam.utils")
    thermo = importlib.import_module("steam.thermodynamics")
    kat_mod = importlib.import_module("tests.test_keyed_noise")
    return sim, noise, utils, thermo, kat_mod


def main(argv):
    import argparse
    ap = argparse.ArgumentParser(description="generate the golden fixtures")
    ap.add_argument("reference", type=Path, help="source tree of thomasdewitt/STEAM")
    ap.add_argument("--part", choices=("unit", "c0", "all"), default="all")
    args = ap.parse_args(argv[1:])
    mods = _import_reference(args.reference)
    if args.part in ("unit", "all"):
        unit_fixtures(*mods)
    if args.part in ("c0", "all"):
        c0_fixtures(*mods)


def c0_fixtures(sim, noise, utils, thermo, kat_mod):
    """The reference's single class step at 128 x 128 x 64."""
    sys.path.insert(0, str(HERE.parent))
    import config_cases as cc

    case = cc.build(sim, cc.C0)
    shape = case['shape']
    idx = cc.sample_index(int(np.prod(shape)))
    fx = {"idx": idx.astype(np.int64), "input_seed": np.int64(2026)}
    zero_comp = [np.ones(shape[2], np.float32)]
    for tshape in ('mexican_hat', 'morlet_omega0_6'):
        tag = 'mh' if tshape == 'mexican_hat' else 'mo'
        h, q, F = cc.inputs(shape)
        out = sim.cascade_loop(
            case['hp'], case['qp'], case['zp'], case['grids'], case['C_h'], case['C_q'],
            case['b_h'], case['b_q'], [case['aspect']], *cc.BOUNDS, 1, (1, 1, 1),
            [case['seed']], h_perturbation=h, qt_perturbation=q, flux=F,
            flux_noise_scale=cc.C1, turbulon_shape=tshape, comp_k=zero_comp)
        h_o, q_o, F_o = out[0], out[1], out[2]
        led = out[7].classes[0]
        hm, qm = case['h_mean'], case['qt_mean']
        diag = thermo.recover_diagnostics(np.clip(h_o + hm, cc.BOUNDS[0], cc.BOUNDS[1]),
                                          np.clip(q_o + qm, cc.BOUNDS[2], cc.BOUNDS[3]),
                                          case['z'], cc.SURFACE_PRESSURE, device='cpu')
        fields = {"flux": F_o, "h": h_o, "qt": q_o, "qc": diag['qc'], "qi": diag['qi'],
                  "T": diag['T']}
        for name, f in fields.items():
            fx[f"{tag}_{name}_sample"] = np.asarray(f).reshape(-1)[idx].astype(np.float32)
            fx[f"{tag}_{name}_levels"] = cc.level_stats(f)
        fl = led.flux
        fx[f"{tag}_flux_ledger"] = np.array([
            fl.entering.total, fl.entering.count, fl.noise_abs.total, fl.noise_abs.count,
            fl.realized.total, fl.realized.count, fl.n_clipped], dtype=np.float64)
        for name in ('h', 'qt'):
            pl = led.pattern[name]
            fx[f"{tag}_{name}_pattern"] = np.stack([np.asarray(pl.level_total, np.float64),
                                                    np.asarray(pl.level_count, np.float64)])
            ba = led.bounded_add[name]
            fx[f"{tag}_{name}_ba_a0"] = np.asarray(ba.a0, np.float64)
            fx[f"{tag}_{name}_ba_mu"] = np.asarray(ba.mu, np.float64)
            fx[f"{tag}_{name}_ba_n_loop"] = np.asarray(ba.n_loop, np.int32)
            fx[f"{tag}_{name}_ba_final_demean"] = np.asarray(ba.final_demean, np.float64)
    out_path = HERE / "c0_class_step.npz"
    np.savez_compressed(out_path, **fx)
    print(f"wrote {out_path} ({out_path.stat().st_size} bytes, {len(fx)} arrays)")


def unit_fixtures(sim, noise, utils, thermo, kat_mod):
    fx = {}

    # -- Philox known answers (Random123 vectors carried by the reference tests)
    kat = kat_mod.PHILOX4X32_10_KAT
    fx["kat_counter"] = np.array([c for c, _, _ in kat], dtype=np.uint64)
    fx["kat_key"] = np.array([k for _, k, _ in kat], dtype=np.uint64)
    fx["kat_out"] = np.array([o for _, _, o in kat], dtype=np.uint64)

    # -- keyed uniforms over an index box with extreme and negative indices
    key = noise.class_key(np.random.SeedSequence(11))
    ix = np.array([0, 1, 2, 7, 100, 2**31 + 5, 2**32 - 1], dtype=np.int64)
    iy = np.array([0, 3, 4096, 2**32 - 2], dtype=np.int64)
    iz = np.array([-3, 0, 1, 2, 3, 255, 70000], dtype=np.int64)
    n = ix.size * iy.size * iz.size
    lane0 = np.empty(n, np.float32)
    lane1 = np.empty(n, np.float32)
    noise.keyed_uniforms(ix, iy, iz, key[0], key[1], key[2], lane0, lane1)
    fx.update(ku_key=np.array(key, dtype=np.uint64), ku_ix=ix, ku_iy=iy, ku_iz=iz,
              ku_lane0=lane0, ku_lane1=lane1)

    # -- CMS transform of those lanes at several alphas
    for a in (1.5, 1.8, 1.95, 2.0):
        fx[f"levy_{a}"] = sim._levy_from_uniforms(a, lane0.copy(), lane1.copy())

    # -- sparse keyed Levy fields: a root, and a wrapped halo region at s > 1
    seeds = np.random.SeedSequence(5).spawn(3)
    r0 = sim.NoiseRegion.root(seeds[0], (8, 6, 5))
    fx["sl_root_key"] = np.array(r0.key, dtype=np.uint64)
    fx["sl_root"] = sim._keyed_sparse_levy((8, 6, 5), (1, 1, 1), 1.8, r0)
    r1 = sim.NoiseRegion(noise.class_key(seeds[1]), (3, 5, 1), (10, 12, 20))
    fx["sl_halo_key"] = np.array(r1.key, dtype=np.uint64)
    fx["sl_halo"] = sim._keyed_sparse_levy((9, 7, 11), (2, 2, 3), 1.8, r1)

    # -- turbulon kernels
    fx["kern_s1"] = sim._turbulon_envelope(1, 0.5, 0.5, 0.5)
    fx["kern_s2"] = sim._turbulon_envelope(1, 0.25, 0.25, 0.25)
    fx["kern_aniso"] = sim._turbulon_envelope(1, 0.5, 0.5, 0.3)
    fx["kern_morlet"] = sim._turbulon_envelope(1, 0.5, 0.5, 0.5, shape='morlet_omega0_6')

    # -- convolution: kernel wider than the field (fold path) and a small
    #    random kernel
    rng = np.random.default_rng(1)
    f1 = rng.standard_normal((12, 10, 9)).astype(np.float32)
    fx["conv1_field"] = f1
    fx["conv1_out"] = utils.convolve_fft_xy_oa_z(f1, fx["kern_s1"], device='cpu')
    f2 = rng.standard_normal((24, 20, 16)).astype(np.float32)
    k2 = rng.standard_normal((5, 7, 3)).astype(np.float32)
    fx["conv2_field"], fx["conv2_kernel"] = f2, k2
    fx["conv2_out"] = utils.convolve_fft_xy_oa_z(f2, k2, device='cpu')
    f3 = rng.standard_normal((32, 28, 24)).astype(np.float32)
    fx["conv3_field"] = f3
    fx["conv3_out"] = utils.convolve_fft_xy_oa_z(f3, fx["kern_s1"], device='cpu')

    # -- flux advance at s=1 (zeroed bottom/top levels) and at s=2
    for tag, shape, sp, kern in (("fa1", (16, 12, 10), (1, 1, 1), fx["kern_s1"]),
                                 ("fa2", (16, 16, 12), (2, 2, 2), fx["kern_s2"])):
        flux = (1.0 + 0.3 * rng.random(shape)).astype(np.float32)
        region = sim.NoiseRegion.root(np.random.SeedSequence(9), shape)
        fx[f"{tag}_flux_in"] = flux.copy()
        fx[f"{tag}_key"] = np.array(region.key, dtype=np.uint64)
        S, led, diag = sim._advance_flux(flux, region, kern, 0.1, 1, sp, n_zero=2,
                                         zero_bottom=True, zero_top=True)
        fx[f"{tag}_S"] = S
        fx[f"{tag}_flux_out"] = flux
        fx[f"{tag}_ledger"] = np.array([
            led.entering.total, led.entering.count, led.noise_abs.total,
            led.noise_abs.count, led.realized.total, led.realized.count,
            led.n_clipped], dtype=np.float64)

    # -- advective weight, uniform and variable dz
    fld = (300e3 + 2e3 * rng.standard_normal((10, 8, 12))).astype(np.float32)
    aspect = (0.2 + rng.random(12)).astype(np.float32)
    z_uni = np.arange(12, dtype=np.float64) * 50.0
    z_var = np.concatenate([[0.0], np.cumsum(40.0 + 15.0 * rng.random(11))])
    fx["aw_field"], fx["aw_aspect"] = fld, aspect
    fx["aw_z_uni"], fx["aw_z_var"] = z_uni, z_var
    fx["aw_uni"] = sim._advective_weight(fld, 100.0, 80.0, z_uni, aspect)
    fx["aw_var"] = sim._advective_weight(fld, 100.0, 80.0, z_var, aspect)
    taper_b = (1e3 + 5e3 * rng.random(12)).astype(np.float32)
    fx["taper_b"] = taper_b
    fx["taper"] = sim._bound_taper(fld.copy(), taper_b, 295e3, 305e3)

    # -- bounded add (host path) with levels pushed against a bound
    nz = 6
    mean = np.linspace(0.0025, 0.012, nz).astype(np.float32)
    pert = (0.002 * rng.standard_normal((14, 12, nz))).astype(np.float32)
    pert = np.clip(pert + mean, 0.0, 0.03).astype(np.float32) - mean
    inc = (0.004 * rng.standard_normal((14, 12, nz))).astype(np.float32)
    fx["ba_pert_in"], fx["ba_mean"], fx["ba_inc_in"] = pert.copy(), mean, inc.copy()
    led = sim._bounded_amplitude_add(pert, mean, inc, 0.0, 0.03, record_applied=True)
    fx["ba_pert_out"], fx["ba_inc_out"] = pert, inc
    fx["ba_a0"], fx["ba_mu"] = led.a0, led.mu

    # -- periodic trilinear regrid
    src = rng.standard_normal((5, 4, 6)).astype(np.float32)
    fx["zoom_src"] = src
    fx["zoom_dyadic"] = utils.zoom_trilinear(src, (10, 8, 9))
    fx["zoom_odd"] = utils.zoom_trilinear(src, (15, 6, 7))

    # -- thermodynamics over a moist column set
    zc = np.arange(20, dtype=np.float64) * 150.0
    hbar = 340e3 - 20e3 * zc / zc[-1]
    qbar = 0.018 - 0.016 * zc / zc[-1]
    h = (hbar + 3e3 * rng.standard_normal((16, 8, 20))).astype(np.float32)
    q = np.clip(qbar + 0.003 * rng.standard_normal((16, 8, 20)), 0, None).astype(np.float32)
    fx["th_h"], fx["th_qt"], fx["th_z"] = h, q, zc
    out = thermo.recover_diagnostics(h, q, zc, 101325.0, device='cpu')
    for k2_, v in out.items():
        fx[f"th_{k2_}"] = v

    # -- grids, amplitude ladder and compensation of a small root run
    zp = np.arange(28) * 30.0
    hp = 340e3 - 20e3 * zp / zp.max()
    qp = 0.018 - 0.016 * zp / zp.max()
    kv = 2000.0 / 2.0 ** np.arange(4)
    grids = sim._compute_all_grids(kv, 2000.0, 2000.0, 800.0, (1, 1, 1),
                                   np.full(28, 100.0), zp)
    for key_ in ('nx', 'ny', 'nz', 'dx', 'dy', 'dz'):
        fx[f"grid_{key_}"] = np.asarray(grids[key_])
    for i, z_i in enumerate(grids['z_arrays']):
        fx[f"grid_z{i}"] = z_i
    kzl = sim._k_z('piecewise_isotropic_below_spheroscale', 2000.0, np.full(28, 100.0))
    C = sim._compute_normalization(hp, zp, kzl, kv, 2000.0, grids)
    for i, c in enumerate(C):
        fx[f"norm_h{i}"] = c
    comp = sim._compensation_profiles(kv, grids['z_arrays'], np.full(28, 100.0), zp,
                                      'piecewise_isotropic_below_spheroscale')
    for i, c in enumerate(comp):
        fx[f"comp{i}"] = c

    # -- a whole small root run (the reference's own fixture configuration)
    captured = {}

    def capture(path, h_3d, qt_3d, *args, **kwargs):
        captured.update(h=h_3d, qt=qt_3d, flux=kwargs.get("flux_3d"))

    sim.write_netcdf = capture
    sim.simulate(h_profile=hp, qt_profile=qp, nx=16, ny=16, dx=125.0, dy=125.0,
                 outer_scale=2000.0, spheroscale=100.0, domain_height=800.0,
                 profile_dz=30.0, output_path=Path(tempfile.mkdtemp()) / "x.nc", seed=42)
    for k3, v in captured.items():
        fx[f"sim_{k3}"] = np.asarray(v)

    np.savez_compressed(OUT, **fx)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(fx)} arrays)")


if __name__ == "__main__":
    main(sys.argv)
