"""Generate tests/golden/reference_fixtures.npz by running the reference.

The reference implementation (thomasdewitt/STEAM, pure Python + numba) is
imported read-only from its source tree -- default /root/reference, or the
path given as the first argument -- with two shims: a one-line ``netCDF4``
import stub (the package imports netCDF4 at module load; nothing here writes
NetCDF) and a scratch NUMBA_CACHE_DIR so that no shipped numba cache is read.

Every fixture is small: inputs and the reference's outputs for the hot-path
stages at toy sizes.  The tests compare the oracle (and, on a GPU, the CUDA
path) against these arrays; the reference itself is never needed at test
time.

Run: python tests/golden/make_golden.py [/path/to/reference]
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
    ref_root = Path(argv[1]) if len(argv) > 1 else Path("/root/reference")
    sim, noise, utils, thermo, kat_mod = _import_reference(ref_root)
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
