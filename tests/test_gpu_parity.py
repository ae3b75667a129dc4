"""CUDA path against the oracle and the reference fixtures (needs a B200).

Tolerances: integer work (Philox, the uniform lattice, the centre lattice) is
bit-exact.  Float64 stages agree with the float64 oracle to 1e-10 relative or
better.  Float32 stages agree with the float64 oracle to a few float32 ulps
per operation; the device's float32 Levy draw uses exactly reduced angles and
is therefore closer to float64 than the reference's own float32 arithmetic,
so float32 comparisons against the reference's float32 fixtures allow the
reference's own error.  The FP32 flux agrees with the FP64 oracle to <= 1e-5
relative L2 in log-flux over positive cells.
"""

import numpy as np
import pytest

from oracle import steam_oracle as O

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (n if n > 0 else 1.0)


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def steam():
    import steam_b200.noise
    import steam_b200.simulate
    import steam_b200.thermodynamics
    import steam_b200.utils
    return steam_b200


# ---------------------------------------------------------------------------
# Keyed noise
# ---------------------------------------------------------------------------

def test_keyed_uniforms_bit_exact(golden, steam):
    key = golden["ku_key"]
    n = golden["ku_lane0"].size
    l0 = np.empty(n, np.float32)
    l1 = np.empty(n, np.float32)
    steam.noise.keyed_uniforms(golden["ku_ix"], golden["ku_iy"], golden["ku_iz"],
                               key[0], key[1], key[2], l0, l1)
    assert np.array_equal(l0.view(np.uint32), golden["ku_lane0"].view(np.uint32))
    assert np.array_equal(l1.view(np.uint32), golden["ku_lane1"].view(np.uint32))


def test_keyed_uniforms_large_box_matches_oracle(steam, torch):
    key = O.class_key(np.random.SeedSequence(123))
    ix = np.arange(0, 40) * 977 + 5
    iy = np.arange(0, 33) * 131
    iz = np.arange(-4, 60)
    n = ix.size * iy.size * iz.size
    l0 = torch.empty(n, dtype=torch.float32, device='cuda')
    l1 = torch.empty(n, dtype=torch.float32, device='cuda')
    steam.noise.keyed_uniforms(torch.as_tensor(ix, device='cuda'),
                               torch.as_tensor(iy, device='cuda'),
                               torch.as_tensor(iz, device='cuda'), *key, l0, l1)
    r0, r1 = O.keyed_uniforms(ix, iy, iz, key)
    assert np.array_equal(l0.cpu().numpy().view(np.uint32), r0.view(np.uint32))
    assert np.array_equal(l1.cpu().numpy().view(np.uint32), r1.view(np.uint32))


def _no_worse_than_reference(got32, ref32, exact64):
    """The device float32 draw is at least as close to the float64 value as
    the reference's own float32 arithmetic is, up to 16 float32 ulps (two
    powf, a logf and three sinpif each contribute a few)."""
    g = got32.astype(np.float64)
    # near a zero of sin(pi alpha v) the float32 product alpha*v alone moves
    # the draw by ~1e-7 of its scale, hence the absolute floor
    floor = 4e-7 * np.sqrt(np.mean(exact64 ** 2))
    bound = np.abs(ref32.astype(np.float64) - exact64) + 16 * np.spacing(
        np.abs(exact64).astype(np.float32)).astype(np.float64) + floor
    assert np.all(np.abs(g - exact64) <= bound)


def test_sparse_levy_fixtures(golden, steam):
    sim = steam.simulate
    k_root = tuple(int(v) for v in golden["sl_root_key"])
    got = sim._keyed_sparse_levy((8, 6, 5), (1, 1, 1), 1.8,
                                 sim.NoiseRegion(k_root, (0, 0, 0), (8, 6, 5)))
    assert np.array_equal(got != 0, golden["sl_root"] != 0)
    exact = O.keyed_sparse_levy((8, 6, 5), (1, 1, 1), 1.8, k_root, dtype=np.float64)
    _no_worse_than_reference(got, golden["sl_root"], exact)
    k_halo = tuple(int(v) for v in golden["sl_halo_key"])
    got = sim._keyed_sparse_levy((9, 7, 11), (2, 2, 3), 1.8,
                                 sim.NoiseRegion(k_halo, (3, 5, 1), (10, 12, 20)))
    assert np.array_equal(got != 0, golden["sl_halo"] != 0)
    exact = O.keyed_sparse_levy((9, 7, 11), (2, 2, 3), 1.8, k_halo, origin=(3, 5, 1),
                                world_shape=(10, 12, 20), dtype=np.float64)
    _no_worse_than_reference(got, golden["sl_halo"], exact)


@pytest.mark.parametrize("alpha", [1.5, 1.8, 1.95, 2.0])
def test_levy_against_float64_oracle(steam, alpha):
    """FP64 device draws equal the FP64 oracle; FP32 device draws (exactly
    reduced angles) are within a few ulps of them, where the reference's own
    float32 arithmetic is off by up to ~1e-2 relative L2."""
    sim = steam.simulate
    shape = (48, 40, 32)
    key = O.class_key(np.random.SeedSequence(77))
    region = sim.NoiseRegion(key, (0, 0, 0), shape)
    want = O.keyed_sparse_levy(shape, (1, 1, 1), alpha, key, dtype=np.float64)
    got = sim._keyed_sparse_levy(shape, (1, 1, 1), alpha, region, dtype=np.float64)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
    got32 = sim._keyed_sparse_levy(shape, (1, 1, 1), alpha, region)
    assert rel_l2(got32, want) < 2e-6
    lit32 = O.keyed_sparse_levy(shape, (1, 1, 1), alpha, key, dtype=np.float32)
    _no_worse_than_reference(got32, lit32, want)


def test_world_restriction_is_exact(steam):
    """A tile's noise is the world's noise restricted to the tile, bit for bit,
    including a halo that wraps around the periodic edge."""
    sim = steam.simulate
    key = O.class_key(np.random.SeedSequence(3))
    world = (32, 24, 12)
    full = sim._keyed_sparse_levy(world, (2, 2, 1), 1.8, sim.NoiseRegion(key, (0, 0, 0), world))
    tile = sim._keyed_sparse_levy((12, 10, 12), (2, 2, 1), 1.8,
                                  sim.NoiseRegion(key, (26, 19, 0), world))
    xs = (26 + np.arange(12)) % 32
    ys = (19 + np.arange(10)) % 24
    assert np.array_equal(tile.view(np.uint32), full[np.ix_(xs, ys)].view(np.uint32))


# ---------------------------------------------------------------------------
# Kernel build
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("name,args,shape", [
    ("kern_s1", (1, 0.5, 0.5, 0.5), "mexican_hat"),
    ("kern_s2", (1, 0.25, 0.25, 0.25), "mexican_hat"),
    ("kern_aniso", (1, 0.5, 0.5, 0.3), "mexican_hat"),
    ("kern_morlet", (1, 0.5, 0.5, 0.5), "morlet_omega0_6"),
])
def test_kernel_build(golden, steam, name, args, shape):
    got = steam.simulate._turbulon_envelope(*args, shape=shape)
    assert got.shape == golden[name].shape
    np.testing.assert_allclose(got, golden[name], rtol=1e-5, atol=2e-6)
    g64 = steam.simulate._turbulon_envelope(*args, shape=shape, dtype=np.float64)
    w64 = O.turbulon_envelope(*args, shape=shape, dtype=np.float64)
    np.testing.assert_allclose(g64, w64, rtol=1e-12, atol=1e-13)


# ---------------------------------------------------------------------------
# Convolution
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("tag,kernel", [("conv1", "kern_s1"), ("conv2", "conv2_kernel"),
                                        ("conv3", "kern_s1")])
def test_convolution_fixtures(golden, steam, tag, kernel):
    got = steam.utils.convolve_fft_xy_oa_z(golden[f"{tag}_field"], golden[kernel])
    assert got.dtype == np.float32
    assert rel_l2(got, golden[f"{tag}_out"]) < 2e-6


@pytest.mark.parametrize("shape", [(40, 36, 30), (7, 9, 20), (64, 48, 5), (33, 17, 70)])
def test_convolution_float64_against_oracle(steam, shape):
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape)
    k = O.turbulon_envelope(1, 0.5, 0.5, 0.5, dtype=np.float64)
    got = steam.utils.convolve_fft_xy_oa_z(f, k)
    assert got.dtype == np.float64
    assert rel_l2(got, O.convolve(f, k)) < 1e-12


def test_convolution_small_full_rank_kernel_float64(steam):
    rng = np.random.default_rng(5)
    f = rng.standard_normal((20, 18, 15))
    k = rng.standard_normal((3, 3, 3))
    got = steam.utils.convolve_fft_xy_oa_z(f, k)
    assert rel_l2(got, O.convolve(f, k)) < 1e-12


def test_convolution_empty_field(steam):
    out = steam.utils.convolve_fft_xy_oa_z(np.zeros((0, 4, 4), np.float32),
                                          np.ones((3, 3, 3), np.float32))
    assert out.shape == (0, 4, 4)


# ---------------------------------------------------------------------------
# Flux advance
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("tag,shape,sp,kern", [("fa1", (16, 12, 10), (1, 1, 1), "kern_s1"),
                                               ("fa2", (16, 16, 12), (2, 2, 2), "kern_s2")])
def test_advance_flux_fixtures(golden, steam, tag, shape, sp, kern):
    sim = steam.simulate
    flux = golden[f"{tag}_flux_in"].copy()
    region = sim.NoiseRegion(tuple(int(v) for v in golden[f"{tag}_key"]), (0, 0, 0), shape)
    S, led, diag = sim._advance_flux(flux, region, golden[kern], 0.1, 1, sp, n_zero=2,
                                     zero_bottom=True, zero_top=True)
    ref = golden[f"{tag}_ledger"]
    assert led.entering.total == pytest.approx(ref[0], rel=1e-12)
    assert led.noise_abs.count == ref[3]
    # the reference's float32 noise carries ~1e-4 relative error of its own
    assert led.noise_abs.total == pytest.approx(ref[2], rel=1e-4)
    assert abs(led.n_clipped - ref[6]) <= 2
    assert rel_l2(S, golden[f"{tag}_S"]) < 2e-4
    assert rel_l2(flux, golden[f"{tag}_flux_out"]) < 1e-4
    # and against the FP64 oracle on the same input, tightly
    f64 = golden[f"{tag}_flux_in"].astype(np.float64)
    kern64 = O.turbulon_envelope(1, 1 / (2 * sp[0]), 1 / (2 * sp[1]), 1 / (2 * sp[2]),
                                 dtype=np.float64)
    S64, _ = O.advance_flux(f64, tuple(int(v) for v in golden[f"{tag}_key"]), kern64, 0.1,
                            1, sp, n_zero=2, zero_bottom=True, zero_top=True)
    assert rel_l2(flux, f64) < 5e-6
    assert rel_l2(S, S64) < 5e-6


def test_advance_flux_float64_against_oracle(steam):
    sim = steam.simulate
    shape = (24, 20, 18)
    rng = np.random.default_rng(8)
    flux0 = 1.0 + 0.3 * rng.random(shape)
    key = O.class_key(np.random.SeedSequence(21))
    kern = O.turbulon_envelope(1, 0.5, 0.5, 0.5, dtype=np.float64)
    f_gpu = flux0.copy()
    S, led, _ = sim._advance_flux(f_gpu, sim.NoiseRegion(key, (0, 0, 0), shape), kern, 0.1,
                                  1, (1, 1, 1), n_zero=2, zero_bottom=True, zero_top=True)
    f_ora = flux0.copy()
    S_o, rec = O.advance_flux(f_ora, key, kern, 0.1, 1, (1, 1, 1), n_zero=2,
                              zero_bottom=True, zero_top=True)
    assert led.n_clipped == rec['n_clipped']
    assert rel_l2(f_gpu, f_ora) < 1e-10
    assert rel_l2(S, S_o) < 1e-10


def _flux_advance_f32(sim, shape, key, k64):
    f32 = np.ones(shape, np.float32)
    sim._advance_flux(f32, sim.NoiseRegion(key, (0, 0, 0), shape), k64, 0.1, 1, (1, 1, 1),
                      n_zero=2, zero_bottom=True, zero_top=True)
    return f32


def test_log_flux_error_float32_vs_float64_oracle(steam):
    """FP32 device flux (float32 convolution arithmetic) against the FP64
    oracle: <= 1e-5 relative L2 in log-flux over the cells clear of the clip
    (F > 1e-3), with an absolute bound on the cells within the clip band and
    the clip masks reported apart.  Over every positive cell, the log of the
    few cells a rounding away from zero dominates (F ~ 1e-5 there): that
    stricter form is held with the flux convolution's float64 accumulation
    (steam_conv_set_flux_wide)."""
    from steam_b200 import _lib
    sim = steam.simulate
    lib = _lib.load()
    shape = (48, 40, 32)
    key = O.class_key(np.random.SeedSequence(99))
    k64 = O.turbulon_envelope(1, 0.5, 0.5, 0.5, dtype=np.float64)
    f64 = np.ones(shape, np.float64)
    O.advance_flux(f64, key, k64, 0.1, 1, (1, 1, 1), n_zero=2, zero_bottom=True,
                   zero_top=True)
    f32 = _flux_advance_f32(sim, shape, key, k64)
    pos = (f64 > 0) & (f32 > 0)
    assert np.count_nonzero((f64 > 0) != (f32 > 0)) <= max(1, pos.size // 10000)
    _log_flux_within(f32, f64, 1e-5)
    try:
        _lib.check(lib.steam_conv_set_flux_wide(1))
        w32 = _flux_advance_f32(sim, shape, key, k64)
    finally:
        _lib.check(lib.steam_conv_set_flux_wide(0))
    pos = (f64 > 0) & (w32 > 0)
    err = rel_l2(np.log(w32[pos].astype(np.float64)), np.log(f64[pos]))
    assert err <= 1e-5, err
    _log_flux_within(w32, f64, 1e-5)


# ---------------------------------------------------------------------------
# Scalar pattern, bounded add, projection
# ---------------------------------------------------------------------------

def test_advective_weight_fixtures(golden, steam):
    for z in ("uni", "var"):
        got = steam.simulate._advective_weight(golden["aw_field"], 100.0, 80.0,
                                               golden[f"aw_z_{z}"], golden["aw_aspect"])
        np.testing.assert_allclose(got, golden[f"aw_{z}"], rtol=2e-5, atol=1e-6)


@pytest.mark.parametrize("dtype,tol", [(np.float32, 2e-5), (np.float64, 1e-11)])
def test_scalar_pattern_against_oracle(steam, torch, dtype, tol):
    sim = steam.simulate
    rng = np.random.default_rng(4)
    shape = (20, 16, 14)
    z = np.concatenate([[0.0], np.cumsum(60.0 + 20.0 * rng.random(13))])
    mean = np.linspace(340e3, 320e3, 14).astype(np.float32)
    pert = (1500.0 * rng.standard_normal(shape)).astype(dtype)
    prod = rng.standard_normal(shape).astype(dtype) * (rng.random(shape) < 0.5)
    aspect = (0.3 + rng.random(14)).astype(np.float32)
    b = (2e3 + 4e3 * rng.random(14)).astype(np.float32)
    C = (100.0 + 50 * rng.random(14)).astype(np.float32)
    s_scale = float(dtype(1.0 / 0.37))
    S = (prod * dtype(s_scale)).astype(dtype)
    Wo, tot, cnt = O.scalar_pattern(pert, mean, S, 100.0, 100.0, z, aspect, b, 315e3, 355e3, C)
    pt = torch.as_tensor(pert, device='cuda')
    W, gtot, gcnt = sim.pattern_device(pt, mean, torch.as_tensor(prod, device='cuda'),
                                       s_scale, 100.0, 100.0, z, aspect, b, 315e3, 355e3)
    assert np.array_equal(gcnt, cnt)
    np.testing.assert_allclose(gtot, tot, rtol=tol)
    lm = (gtot / np.maximum(gcnt, 1)).astype(dtype)
    Wn = (W.cpu().numpy() / np.where(lm > 0, lm, 1)[None, None, :]) * C[None, None, :]
    assert rel_l2(Wn, Wo) < tol * 10


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_bounded_add_against_oracle(golden, steam, dtype):
    sim = steam.simulate
    pert = golden["ba_pert_in"].astype(dtype)
    inc = golden["ba_inc_in"].astype(dtype)
    p_o, i_o = pert.copy(), inc.copy()
    rec = O.bounded_amplitude_add(p_o, golden["ba_mean"], i_o, 0.0, 0.03, record_applied=True)
    p_g, i_g = pert.copy(), inc.copy()
    led = sim._bounded_amplitude_add(p_g, golden["ba_mean"], i_g, 0.0, 0.03,
                                     record_applied=True)
    atol = 2e-9 if dtype == np.float32 else 1e-13
    np.testing.assert_allclose(p_g, p_o, rtol=0, atol=atol)
    np.testing.assert_allclose(i_g, i_o, rtol=0, atol=atol)
    np.testing.assert_allclose(led.a0, rec['a0'], rtol=1e-10)
    if dtype == np.float32:
        np.testing.assert_allclose(p_g, golden["ba_pert_out"], rtol=0, atol=atol)
    # the three deposit conditions: bounds, zero level mean
    field = p_g + golden["ba_mean"][None, None, :].astype(dtype)
    assert field.min() >= -1e-9 and field.max() <= 0.03 + 1e-9
    assert np.all(np.abs(i_g.mean(axis=(0, 1))) < 1e-6 * np.maximum(led.a0, 1e-30) + 1e-12)


def test_bounded_add_larger_levels(steam):
    """Many levels, some against each bound, some interior, a clip-only level."""
    sim = steam.simulate
    rng = np.random.default_rng(12)
    nz = 40
    shape = (64, 48, nz)
    mean = np.linspace(0.0005, 0.029, nz).astype(np.float32)
    pert = np.clip(0.003 * rng.standard_normal(shape) + mean, 0, 0.03).astype(np.float32) - mean
    inc = (0.005 * rng.standard_normal(shape)).astype(np.float32)
    inc[:, :, 7] = 0.0
    p_o, i_o = pert.copy(), inc.copy()
    O.bounded_amplitude_add(p_o, mean, i_o, 0.0, 0.03, record_applied=True)
    p_g, i_g = pert.copy(), inc.copy()
    led = sim._bounded_amplitude_add(p_g, mean, i_g, 0.0, 0.03, record_applied=True)
    # the device solver stops once the shift is bracketed to a0 2^-20 (the
    # float32 staircase of the level mean); a cell then differs by at most
    # that plus a rounding at each end
    atol = np.ldexp(float(np.max(led.a0)), -20) + 2 * float(np.spacing(np.float32(0.03)))
    np.testing.assert_allclose(p_g, p_o, rtol=0, atol=atol)


def test_projection_against_oracle(steam):
    sim = steam.simulate
    rng = np.random.default_rng(6)
    shape = (30, 20, 12)
    mean = np.linspace(0.001, 0.02, 12).astype(np.float32)
    pert = (0.004 * rng.standard_normal(shape)).astype(np.float32)
    p_o = pert.copy()
    mu_o = O.project_onto_bounds(p_o, mean, 0.0, 0.03)
    p_g = pert.copy()
    led = sim._project_onto_bounds(p_g, mean, 0.0, 0.03)
    assert np.array_equal(np.isnan(led.mu), np.isnan(mu_o))
    np.testing.assert_allclose(p_g, p_o, rtol=0, atol=2e-9)


# ---------------------------------------------------------------------------
# Regrid, thermodynamics
# ---------------------------------------------------------------------------

def test_zoom_fixtures(golden, steam):
    np.testing.assert_allclose(steam.utils.zoom_trilinear(golden["zoom_src"], (10, 8, 9)),
                               golden["zoom_dyadic"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(steam.utils.zoom_trilinear(golden["zoom_src"], (15, 6, 7)),
                               golden["zoom_odd"], rtol=1e-5, atol=1e-6)


def test_thermodynamics_fixtures(golden, steam):
    out = steam.thermodynamics.recover_diagnostics(golden["th_h"], golden["th_qt"],
                                                    golden["th_z"], 101325.0)
    np.testing.assert_allclose(out["T"], golden["th_T"], rtol=0, atol=2e-3)
    np.testing.assert_allclose(out["p"], golden["th_p"], rtol=2e-6)
    for k in ("qv", "qc", "qi"):
        np.testing.assert_allclose(out[k], golden[f"th_{k}"], rtol=0, atol=2e-7)


def test_thermodynamics_float64_against_oracle(golden, steam):
    h = golden["th_h"].astype(np.float64)
    q = golden["th_qt"].astype(np.float64)
    out = steam.thermodynamics.recover_diagnostics(h, q, golden["th_z"], 101325.0)
    want = O.recover_diagnostics(h, q, golden["th_z"], 101325.0)
    for k in ("T", "qv", "qc", "qi", "p"):
        np.testing.assert_allclose(out[k], want[k], rtol=1e-10, atol=1e-14)


# ---------------------------------------------------------------------------
# One class of the cascade, and a whole small run
# ---------------------------------------------------------------------------

def _one_class_setup(nx=32, ny=24, nz=20):
    from steam_b200 import simulate as sim
    zp = np.arange(64) * 50.0
    hp = (340e3 - 20e3 * zp / zp.max()).astype(np.float32)
    qp = (0.018 - 0.016 * zp / zp.max()).astype(np.float32)
    k = 200.0
    grids = sim._compute_all_grids(np.array([k]), nx * 100.0, ny * 100.0, nz * 100.0,
                                   (1, 1, 1), np.full(64, 1000.0), zp)
    assert (grids['nx'][0], grids['ny'][0], grids['nz'][0]) == (nx, ny, nz)
    kzl = sim._k_z('piecewise_isotropic_below_spheroscale', 12800.0, np.full(64, 1000.0))
    C_h = sim._compute_normalization(hp, zp, kzl, np.array([k]), 12800.0, grids)
    C_q = sim._compute_normalization(qp, zp, kzl, np.array([k]), 12800.0, grids)
    return sim, zp, hp, qp, grids, C_h, C_q


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_single_class_step_against_oracle(steam, dtype):
    sim, zp, hp, qp, grids, C_h, C_q = _one_class_setup()
    b_h = sim._bound_buffers(C_h, 1)
    b_q = sim._bound_buffers(C_q, 1)
    aspect = [np.ones(20, np.float32)]
    seeds = np.random.SeedSequence(0).spawn(1)
    rng = np.random.default_rng(0)
    shape = (32, 24, 20)
    h0 = (800.0 * rng.standard_normal(shape)).astype(dtype)
    q0 = (0.0008 * rng.standard_normal(shape)).astype(dtype)
    F0 = (1.0 + 0.2 * rng.random(shape)).astype(dtype)
    out = sim.cascade_loop(hp, qp, zp, grids, C_h, C_q, b_h, b_q, aspect, 315 * 1004,
                           355 * 1004, 0.0, 0.03, 1, (1, 1, 1), seeds,
                           h_perturbation=h0, qt_perturbation=q0, flux=F0,
                           comp_k=[np.ones(20, np.float32)], dtype=dtype)
    h_g, q_g, F_g = out[0], out[1], out[2]
    z = grids['z_arrays'][0]
    key = O.class_key(seeds[0])
    kern = O.turbulon_envelope(1, 0.5, 0.5, 0.5, dtype=np.float64)
    h_o, q_o, F_o = (a.astype(np.float64) for a in (h0, q0, F0))
    O.class_step(h_o, q_o, F_o, key, kern,
                 h_mean=np.interp(z, zp, hp).astype(np.float32),
                 qt_mean=np.interp(z, zp, qp).astype(np.float32), z_coords=z,
                 dx=100.0, dy=100.0, aspect=aspect[0], C_h=C_h[0], C_qt=C_q[0], b_h=b_h[0],
                 b_qt=b_q[0], h_min=315 * 1004, h_max=355 * 1004, qt_min=0.0, qt_max=0.03,
                 flux_noise_scale=sim.FLUX_SCALE, n_per_dyad=1, sparsity_factors=(1, 1, 1),
                 n_zero=2)
    tol = 1e-9 if dtype == np.float64 else 1e-5
    assert rel_l2(F_g, F_o) < tol
    assert rel_l2(h_g - h0, h_o - h0) < tol * 10
    assert rel_l2(q_g - q0, q_o - q0) < tol * 10
    _log_flux_within(F_g, F_o, tol)


def _log_flux_within(F_g, F_o, tol, clip_band=1e-3):
    """log-flux relative L2 over cells clear of the clip, and an absolute
    bound on the cells within ``clip_band`` of it.  Where F + conv nearly
    cancels, float32 storage of the noise alone moves log F by O(1) relative
    to O(1e-6) values, so those cells are held to an absolute flux bound
    (reported apart, as the clip mask is)."""
    F_g = F_g.astype(np.float64)
    clear = (F_o > clip_band) & (F_g > clip_band)
    assert rel_l2(np.log(F_g[clear]), np.log(F_o[clear])) < tol
    both_clipped = (F_o == 0) & (F_g == 0)
    near = ~clear & ~both_clipped
    assert np.count_nonzero(near) < max(8, F_o.size // 100)
    if np.any(near):
        assert np.max(np.abs(F_g[near] - F_o[near])) < 20 * tol * clip_band


def test_small_root_run_statistics(golden, steam):
    """A whole 16 x 16 root run (4 classes) against the reference's own run of
    the same configuration.  The cascade's clip and bounded add amplify
    roundoff, so the comparison is statistical: level means and spreads."""
    sim = steam.simulate
    zp = np.arange(28) * 30.0
    hp = 340e3 - 20e3 * zp / zp.max()
    qp = 0.018 - 0.016 * zp / zp.max()
    res = sim.simulate(h_profile=hp, qt_profile=qp, nx=16, ny=16, dx=125.0, dy=125.0,
                       outer_scale=2000.0, spheroscale=100.0, domain_height=800.0,
                       profile_dz=30.0, output_path=None, seed=42)
    for name, span in (("h", 40 * 1004), ("qt", 0.03)):
        got, ref = res[name], golden[f"sim_{name}"]
        assert got.shape == ref.shape
        lm_g = got.mean(axis=(0, 1))
        lm_r = ref.mean(axis=(0, 1))
        assert np.max(np.abs(lm_g - lm_r)) < 1e-3 * span
        sd_g, sd_r = got.std(axis=(0, 1)), ref.std(axis=(0, 1))
        assert np.max(np.abs(sd_g - sd_r) / np.maximum(sd_r, 1e-12 * span)) < 0.25
    assert res["flux"].mean() == pytest.approx(golden["sim_flux"].mean(), rel=1e-3)


def test_repeat_runs_are_bit_identical(steam):
    sim = steam.simulate
    key = O.class_key(np.random.SeedSequence(17))
    kern = O.turbulon_envelope(1, 0.5, 0.5, 0.5)
    outs = []
    for _ in range(2):
        f = np.ones((40, 32, 24), np.float32)
        S, led, _ = sim._advance_flux(f, sim.NoiseRegion(key, (0, 0, 0), f.shape), kern, 0.1,
                                      1, (1, 1, 1))
        outs.append((f, S, led.realized.total))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]


# ---------------------------------------------------------------------------
# Resident (asynchronous) class step against the stage-by-stage step
# ---------------------------------------------------------------------------

def _resident_case(dtype, shape, window):
    import torch
    from steam_b200 import simulate as sim
    from steam_b200.ledger import ClassLedger
    from steam_b200.resident import ResidentClass
    nx, ny, nz = shape
    sim_, zp, hp, qp, grids, C_h, C_q = _one_class_setup(nx, ny, nz)
    b_h = sim._bound_buffers(C_h, 1)[0]
    b_q = sim._bound_buffers(C_q, 1)[0]
    key = O.class_key(np.random.SeedSequence(5))
    setup = sim.make_class_setup(
        grids, 0, h_profile=hp, qt_profile=qp, z_profile=zp, C_h=C_h[0], C_qt=C_q[0],
        b_h=b_h, b_qt=b_q, aspect=np.ones(nz, np.float32),
        bounds=(315 * 1004.0, 355 * 1004.0, 0.0, 0.03), key=key, flux_noise_scale=0.1,
        window=window, dtype=dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    rng = np.random.default_rng(3)
    h0 = torch.as_tensor(800.0 * rng.standard_normal(shape), dtype=tdt, device='cuda')
    q0 = torch.as_tensor(0.0008 * rng.standard_normal(shape), dtype=tdt, device='cuda')
    F0 = torch.as_tensor(1.0 + 0.2 * rng.random(shape), dtype=tdt, device='cuda')
    # stage by stage, every scalar through the host
    hs, qs, Fs = h0.clone(), q0.clone(), F0.clone()
    cl_s = ClassLedger()
    sim.run_class(hs, qs, Fs, None, None, None, setup, cl_s, resident=False)
    # resident: two steps in a row from the same state (the second reuses
    # every resident buffer)
    rc = ResidentClass(setup, tdt)
    for _ in range(2):
        hr, qr, Fr = h0.clone(), q0.clone(), F0.clone()
        rc.step(hr, qr, Fr)
        cl_r = rc.class_ledger()
    return (hs, qs, Fs, cl_s), (hr, qr, Fr, cl_r)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape,window", [((32, 24, 20), None), ((40, 32, 16), (4, 36, 2, 30))])
def test_resident_step_matches_stage_by_stage(steam, dtype, shape, window):
    (hs, qs, Fs, cl_s), (hr, qr, Fr, cl_r) = _resident_case(dtype, shape, window)
    # identical arithmetic, so identical bits
    for a, b in ((hs, hr), (qs, qr), (Fs, Fr)):
        assert bool((a == b).all()), float((a - b).abs().max())
    fs, fr = cl_s.flux, cl_r.flux
    for name in ('entering', 'noise_abs', 'realized'):
        assert getattr(fs, name).total == getattr(fr, name).total
        assert getattr(fs, name).count == getattr(fr, name).count
    assert fs.n_clipped == fr.n_clipped
    for name in ('h', 'qt'):
        np.testing.assert_array_equal(cl_s.pattern[name].level_total,
                                      cl_r.pattern[name].level_total)
        np.testing.assert_array_equal(cl_s.pattern[name].level_count,
                                      cl_r.pattern[name].level_count)
        bs, br = cl_s.bounded_add[name], cl_r.bounded_add[name]
        np.testing.assert_array_equal(bs.a0, br.a0)
        np.testing.assert_array_equal(bs.n_loop, br.n_loop)
        np.testing.assert_array_equal(bs.final_demean, br.final_demean)
        np.testing.assert_array_equal(bs.mu, br.mu)
        assert bs.n_sweeps == br.n_sweeps


def test_field_step_pipelined_steps_match_resident_steps(steam):
    """field_step with wait=False, three steps in a row on the same page-locked
    arrays (each step's uploads overlapping the previous step's downloads),
    gives the bits and ledgers of three resident steps on device tensors."""
    import torch
    from steam_b200 import simulate as sim
    from steam_b200.resident import ResidentClass
    nx, ny, nz = 32, 24, 20
    sim_, zp, hp, qp, grids, C_h, C_q = _one_class_setup(nx, ny, nz)
    setup = sim.make_class_setup(
        grids, 0, h_profile=hp, qt_profile=qp, z_profile=zp, C_h=C_h[0], C_qt=C_q[0],
        b_h=sim._bound_buffers(C_h, 1)[0], b_qt=sim._bound_buffers(C_q, 1)[0],
        aspect=np.ones(nz, np.float32), bounds=(315 * 1004.0, 355 * 1004.0, 0.0, 0.03),
        key=O.class_key(np.random.SeedSequence(9)), flux_noise_scale=0.1, dtype=np.float32)
    rng = np.random.default_rng(6)

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        t.copy_(torch.from_numpy(a))
        return t.numpy()
    h = pinned((800.0 * rng.standard_normal((nx, ny, nz))).astype(np.float32))
    q = pinned((0.0008 * rng.standard_normal((nx, ny, nz))).astype(np.float32))
    F = pinned((1.0 + 0.2 * rng.random((nx, ny, nz))).astype(np.float32))
    ht, qt_, Ft = (torch.as_tensor(a.copy(), device='cuda') for a in (h, q, F))
    rc = ResidentClass(setup, torch.float32)
    want = []
    for _ in range(3):
        diag = {k: torch.empty_like(ht) for k in ("T", "qv", "qc", "qi", "p")}
        rc.step(ht, qt_, Ft, diagnostics=diag)
        want.append((diag["qc"].cpu().numpy(), diag["qi"].cpu().numpy(),
                     rc.class_ledger().flux.realized.total))
    outs = [{k: pinned(np.zeros((nx, ny, nz), np.float32)) for k in ("qc", "qi")}
            for _ in range(3)]
    pend = [sim.field_step(h, q, F, setup, out=o, wait=False) for o in outs]
    got = [p.result() for p in pend]
    for (d, led), (qc, qi, realized) in zip(got, want):
        np.testing.assert_array_equal(d["qc"], qc)
        np.testing.assert_array_equal(d["qi"], qi)
        assert led.flux.realized.total == realized
    np.testing.assert_array_equal(h, ht.cpu().numpy())
    np.testing.assert_array_equal(q, qt_.cpu().numpy())
    np.testing.assert_array_equal(F, Ft.cpu().numpy())


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_field_step_host_arrays_match_resident_tensors(steam, dtype):
    """field_step on numpy arrays (pipelined copies on a second stream) gives
    the same bits as the resident step on device tensors, twice in a row."""
    import torch
    from steam_b200 import simulate as sim
    from steam_b200.resident import ResidentClass
    nx, ny, nz = 32, 24, 20
    sim_, zp, hp, qp, grids, C_h, C_q = _one_class_setup(nx, ny, nz)
    setup = sim.make_class_setup(
        grids, 0, h_profile=hp, qt_profile=qp, z_profile=zp, C_h=C_h[0], C_qt=C_q[0],
        b_h=sim._bound_buffers(C_h, 1)[0], b_qt=sim._bound_buffers(C_q, 1)[0],
        aspect=np.ones(nz, np.float32), bounds=(315 * 1004.0, 355 * 1004.0, 0.0, 0.03),
        key=O.class_key(np.random.SeedSequence(9)), flux_noise_scale=0.1, dtype=dtype)
    rng = np.random.default_rng(4)
    h = (800.0 * rng.standard_normal((nx, ny, nz))).astype(dtype)
    q = (0.0008 * rng.standard_normal((nx, ny, nz))).astype(dtype)
    F = (1.0 + 0.2 * rng.random((nx, ny, nz))).astype(dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    ht, qt_, Ft = (torch.as_tensor(a, device='cuda') for a in (h, q, F))
    rc = ResidentClass(setup, tdt)
    for _ in range(2):
        diag = {k: torch.empty_like(ht) for k in ("T", "qv", "qc", "qi", "p")}
        rc.step(ht, qt_, Ft, diagnostics=diag)
        out = {k: torch.empty((nx, ny, nz), dtype=tdt, pin_memory=True).numpy()
               for k in ("qc",)}
        got, _ = sim.field_step(h, q, F, setup, diagnostics=("qc", "qi"), out=out)
        np.testing.assert_array_equal(h, ht.cpu().numpy())
        np.testing.assert_array_equal(q, qt_.cpu().numpy())
        np.testing.assert_array_equal(F, Ft.cpu().numpy())
        np.testing.assert_array_equal(got["qc"], diag["qc"].cpu().numpy())
        np.testing.assert_array_equal(got["qi"], diag["qi"].cpu().numpy())
        assert got["qc"] is out["qc"] or np.shares_memory(got["qc"], out["qc"])
