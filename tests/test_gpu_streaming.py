"""streamed_cascade_loop and simulate(stream_to_disk=True): the resident
cascade delivered through the z-major scratch store gives the same fields as
the plain run, and the store leaves nothing behind."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ZP = np.arange(28) * 30.0
HP = 340e3 - 20e3 * ZP / ZP.max()
QP = 0.018 - 0.016 * ZP / ZP.max()
ARGS = dict(h_profile=HP, qt_profile=QP, nx=16, ny=16, dx=125.0, dy=125.0,
            outer_scale=2000.0, spheroscale=100.0, domain_height=800.0, profile_dz=30.0,
            output_path=None, seed=42)


def test_simulate_streamed_equals_resident(tmp_path):
    from steam_b200 import simulate as sim
    plain = sim.simulate(**ARGS)
    streamed = sim.simulate(**ARGS, stream_to_disk=True, scratch_dir=tmp_path)
    for k in ("h", "qt", "flux"):
        np.testing.assert_array_equal(streamed[k], plain[k])
    assert not any(tmp_path.rglob("*.npy"))  # the store was destroyed


def test_streamed_cascade_loop_store(tmp_path):
    from steam_b200 import simulate as sim
    from steam_b200.streaming import plan_tiling, streamed_cascade_loop
    # the cascade's inputs as simulate builds them
    res = sim.simulate(**ARGS, resident=True)
    grids = res["grids"]
    n = len(grids["k"])
    C_h = sim._compute_normalization(np.float32(HP), ZP, sim._k_z(
        'piecewise_isotropic_below_spheroscale', 2000.0, np.full(ZP.size, 100.0)),
        grids["k"], 2000.0, grids)
    C_q = sim._compute_normalization(np.float32(QP), ZP, sim._k_z(
        'piecewise_isotropic_below_spheroscale', 2000.0, np.full(ZP.size, 100.0)),
        grids["k"], 2000.0, grids)
    aspect = [np.ones(int(grids["nz"][i]), np.float32) for i in range(n)]
    b_h = sim._bound_buffers(C_h, 1)
    b_q = sim._bound_buffers(C_q, 1)
    seeds = np.random.SeedSequence(42).spawn(n)
    args = (np.float32(HP), np.float32(QP), ZP, grids, C_h, C_q, b_h, b_q, aspect,
            315 * 1004, 355 * 1004, 0.0, 0.03, 1, (1, 1, 1), seeds)
    ref = sim.cascade_loop(*args, comp_k=None)
    plan = plan_tiling(grids, (13, 13, 13), budget_bytes=1 << 34)
    assert plan.horizon == n and plan.halo == (7, 7)
    out = streamed_cascade_loop(*args, plan, tmp_path)
    store = out[-1]
    for got, want in zip(out[:3], ref[:3]):
        np.testing.assert_array_equal(np.asarray(got), want)
    raw = np.load(store.path(n - 1, "flux"), mmap_mode="r")
    assert raw.shape == (ref[2].shape[2], ref[2].shape[0], ref[2].shape[1])  # z-major
    store.destroy()
    assert not (tmp_path / "steam_b200_store").exists()
