"""Host-side logic and the C ABI, without a GPU."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib
from steam_b200 import simulate as S
from steam_b200 import utils as U

REPO = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (REPO / "include" / "steam_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(steam_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = header_symbols()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(_lib.exported_symbols()) == declared
    assert lib.steam_version() >= 1


def test_error_path_without_device_work():
    lib = _lib.load()
    rc = lib.steam_keyed_uniforms(None, -1, None, 0, None, 0, 0, 0, 0, None, None, None)
    assert rc == 1
    assert b"negative" in lib.steam_last_error()
    with pytest.raises(ValueError):
        _lib.check(rc)


def test_grids_match_reference(golden):
    zp = np.arange(28) * 30.0
    kv = 2000.0 / 2.0 ** np.arange(4)
    g = S._compute_all_grids(kv, 2000.0, 2000.0, 800.0, (1, 1, 1), np.full(28, 100.0), zp)
    for key in ('nx', 'ny', 'nz'):
        assert np.array_equal(g[key], golden[f"grid_{key}"])
    for key in ('dx', 'dy', 'dz'):
        np.testing.assert_allclose(g[key], golden[f"grid_{key}"], rtol=1e-14)
    for i, z in enumerate(g['z_arrays']):
        np.testing.assert_allclose(z, golden[f"grid_z{i}"], rtol=1e-13, atol=1e-9)


def test_normalization_and_compensation_match_reference(golden):
    zp = np.arange(28) * 30.0
    hp = 340e3 - 20e3 * zp / zp.max()
    kv = 2000.0 / 2.0 ** np.arange(4)
    sph = np.full(28, 100.0)
    g = S._compute_all_grids(kv, 2000.0, 2000.0, 800.0, (1, 1, 1), sph, zp)
    kzl = S._k_z('piecewise_isotropic_below_spheroscale', 2000.0, sph)
    C = S._compute_normalization(hp, zp, kzl, kv, 2000.0, g)
    for i, c in enumerate(C):
        np.testing.assert_allclose(c, golden[f"norm_h{i}"], rtol=1e-6)
    comp = S._compensation_profiles(kv, g['z_arrays'], sph, zp,
                                    'piecewise_isotropic_below_spheroscale')
    for i, c in enumerate(comp):
        np.testing.assert_allclose(c, golden[f"comp{i}"], rtol=1e-7)


@pytest.mark.parametrize("k,n", [(13, 12), (13, 10), (13, 13), (13, 7), (13, 6), (5, 24)])
def test_effective_centre_reproduces_fold(k, n):
    """The modular convolution with the effective centre equals the reference's
    fold-then-centre convolution, on odd and even periods."""
    rng = np.random.default_rng(k * 100 + n)
    f = rng.standard_normal((n, 3, 4))
    kern = rng.standard_normal((k, 1, 1))
    want = O.convolve(f, kern)
    c = U.effective_centre(k, n)
    got = np.zeros_like(f)
    for x in range(n):
        for i in range(k):
            got[x] += kern[i, 0, 0] * f[(x - i + c) % n]
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-10)


def test_factorisation_of_turbulon_kernels(golden):
    for name, tol in (("kern_s1", 1e-6), ("kern_s2", 1e-6), ("kern_aniso", 1e-6)):
        Px, Py, Pz, core, err = U.factor_kernel(golden[name], tol)
        assert (Px.shape[1], Py.shape[1], Pz.shape[1]) == (2, 2, 2)
        assert err < tol
    k64 = O.turbulon_envelope(1, 0.5, 0.5, 0.5, dtype=np.float64)
    Px, Py, Pz, core, err = U.factor_kernel(k64, 1e-12)
    assert (Px.shape[1], Py.shape[1], Pz.shape[1]) == (2, 2, 2)
    assert err < 1e-12
    plan = U.plan_convolution(golden["kern_s1"], (64, 64, 32), np.float32)
    assert plan.kind == 'separable' and plan.spec.n_pairs == 4
    rnd = np.random.default_rng(3).standard_normal((7, 7, 7))
    assert U.plan_convolution(rnd, (16, 16, 16), np.float32).kind == 'fft'
    assert U.plan_convolution(rnd, (16, 16, 16), np.float64).kind == 'direct'
    morlet = O.turbulon_envelope(1, 0.5, 0.5, 0.5, shape='morlet_omega0_6', dtype=np.float64)
    # the Morlet turbulon factors to Tucker rank 3 at float32 tolerance, beyond
    # the fused separable kernel: the FFT form; at float64 tolerance it does not
    assert U.plan_convolution(morlet, (64, 64, 32), np.float32).kind == 'fft'
    assert U.plan_convolution(morlet, (64, 64, 32), np.float64).kind == 'direct'
    wide = np.random.default_rng(4).standard_normal((27, 5, 5))
    p = U.plan_convolution(wide, (16, 16, 16), np.float32)
    assert p.kind == 'direct' and p.centre == (U.effective_centre(27, 16), 2)


def test_turbulon_plan_has_three_filter_pairs():
    """A float64 turbulon kernel, a sum of separable terms
    g g g (3 - x^2 - y^2 - z^2), gets y and z bases in which one of the four
    (z filter, y filter) pairs vanishes; the 3-pair network still equals the
    kernel to roundoff.  A float32-rounded kernel keeps all four pairs."""
    for args in ((1, 0.5, 0.5, 0.5), (1, 0.5, 0.5, 0.25), (2, 0.5, 0.5, 0.5)):
        K = O.turbulon_envelope(*args, dtype=np.float64)
        plan = U.plan_convolution(K, (64, 64, 32), np.float64)
        sp = plan.spec
        assert plan.kind == 'separable' and sp.n_pairs == 3
        assert sorted((sp.pair_z[q], sp.pair_y[q]) for q in range(3)) == [(0, 0), (0, 1), (1, 0)]
        Z = np.ctypeslib.as_array(plan.z_taps)[:sp.n_z * sp.kz].reshape(sp.n_z, sp.kz)
        Y = np.ctypeslib.as_array(plan.y_taps)[:sp.n_y * sp.ky].reshape(sp.n_y, sp.ky)
        X = np.ctypeslib.as_array(plan.x_taps)[:sp.n_x * sp.kx].reshape(sp.n_x, sp.kx)
        rec = np.zeros_like(K)
        for a in range(sp.n_x):
            for q in range(sp.n_pairs):
                rec += sp.mix[a * sp.n_pairs + q] * np.einsum(
                    'i,j,k->ijk', X[a], Y[sp.pair_y[q]], Z[sp.pair_z[q]])
        assert np.linalg.norm(rec - K) / np.linalg.norm(K) < 1e-12


def test_separable_plan_reconstructs_kernel(golden):
    """The separable network given to the device equals the kernel."""
    K = golden["kern_s1"].astype(np.float64)
    plan = U.plan_convolution(K, (64, 64, 32), np.float32)
    sp = plan.spec
    Z = np.ctypeslib.as_array(plan.z_taps)[:sp.n_z * sp.kz].reshape(sp.n_z, sp.kz)
    Y = np.ctypeslib.as_array(plan.y_taps)[:sp.n_y * sp.ky].reshape(sp.n_y, sp.ky)
    X = np.ctypeslib.as_array(plan.x_taps)[:sp.n_x * sp.kx].reshape(sp.n_x, sp.kx)
    rec = np.zeros_like(K)
    for a in range(sp.n_x):
        for q in range(sp.n_pairs):
            m = sp.mix[a * sp.n_pairs + q]
            rec += m * np.einsum('i,j,k->ijk', X[a], Y[sp.pair_y[q]], Z[sp.pair_z[q]])
    assert np.linalg.norm(rec - K) / np.linalg.norm(K) < 1e-6


def test_tile_store_owns_only_its_subtree(tmp_path):
    from steam_b200.streaming import TileStore
    st = TileStore(tmp_path)
    raw = st.create(0, "h", (4, 3, 5))
    raw[...] = np.arange(60, dtype=np.float32).reshape(5, 4, 3)
    view = st.open(0, "h")
    assert view.shape == (4, 3, 5) and view[1, 2, 3] == raw[3, 1, 2]
    (tmp_path / "keep.txt").write_text("caller data")
    st.destroy()
    assert (tmp_path / "keep.txt").exists() and not st.root.exists()
    foreign = tmp_path / "foreign"
    foreign.mkdir()
    (foreign / "x").write_text("x")
    with pytest.raises(OSError):
        TileStore(tmp_path, owned_root=foreign)


def test_plan_tiling_halo_and_budget():
    from steam_b200.streaming import plan_tiling
    grids = {'k': np.array([400.0, 200.0]), 'nx': np.array([64, 128]),
             'ny': np.array([64, 128]), 'nz': np.array([32, 64])}
    plan = plan_tiling(grids, (37, 13, 13), budget_bytes=1 << 40)
    assert plan.horizon == 2 and plan.halo == (19, 7) and plan.tiles == {}
    forced = plan_tiling(grids, (13, 13, 13), force=(1, 2, 2))
    assert forced.horizon == 1 and forced.tiles == {1: (2, 2)}
    with pytest.raises(MemoryError):
        plan_tiling(grids, (13, 13, 13), budget_bytes=1000)


def test_tile_server_refuses_oversize_and_bad_requests_before_a_slot():
    """A request larger than the server's max_n, or outside the world's z
    range, is a ValueError at admission; the budget count is untouched."""
    from types import SimpleNamespace

    from steam_b200 import serving

    world = SimpleNamespace(shape=(64, 64, 32), n_zero=2)
    world.tile_box = lambda origin, n: serving.TileWorld.tile_box(world, origin, n)
    server = SimpleNamespace(max_n=16, world=world, in_flight_bytes=0)
    check = serving.TileServer.check_request
    check(server, {'origin': (0, 0, 0), 'n': 16})
    with pytest.raises(ValueError, match="max_n"):
        check(server, {'origin': (0, 0, 0), 'n': 32})
    with pytest.raises(ValueError, match="outside"):
        check(server, {'origin': (0, 0, 20), 'n': 16})
    assert server.in_flight_bytes == 0
