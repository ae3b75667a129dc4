"""Apply-only ledger replay on the device (needs a B200).

The reference's measure/apply split (steam/ledger.py:145-209,
steam/simulate.py:864-870, 3196-3213, 3462-3488, and its bit-exact replay
test, tests/test_measure_apply.py:207-296): a recorded ledger replays a
solve with no reduction at all, to the same bits -- on the whole field, and
on any subset of its columns (what a tile of the world is).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ba_case(shape, seed=3, dtype=np.float32):
    rng = np.random.default_rng(seed)
    nz = shape[2]
    mean = np.linspace(0.0025, 0.012, nz).astype(np.float32)
    pert = (0.002 * rng.standard_normal(shape)).astype(dtype)
    pert = (np.clip(pert + mean, 0.0, 0.03) - mean).astype(dtype)
    inc = (0.004 * rng.standard_normal(shape)).astype(dtype)
    return pert, mean, inc


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(40, 36, 16), (30, 22, 6), (96, 80, 32)])
def test_bounded_add_replay_is_bit_exact(dtype, shape):
    from steam_b200 import simulate as sim
    pert, mean, inc = _ba_case(shape, dtype=dtype)
    p_solve, i_solve = pert.copy(), inc.copy()
    led = sim._bounded_amplitude_add(p_solve, mean, i_solve, 0.0, 0.03, record_applied=True)
    assert led.n_sweeps > 0 and np.any(led.n_loop > 0) and np.any(led.bisected)
    # the whole field
    p_rep, i_rep = pert.copy(), inc.copy()
    out = sim._bounded_amplitude_add(p_rep, mean, i_rep, 0.0, 0.03, record_applied=True,
                                     ledger=led)
    assert out is led
    np.testing.assert_array_equal(p_rep, p_solve)
    np.testing.assert_array_equal(i_rep, i_solve)
    # a tile of its columns, on its own
    sl = (slice(7, 29), slice(3, 17))
    p_t = np.ascontiguousarray(pert[sl])
    sim._bounded_amplitude_add(p_t, mean, np.ascontiguousarray(inc[sl]), 0.0, 0.03,
                               ledger=led)
    np.testing.assert_array_equal(p_t, p_solve[sl])


def test_bounded_add_ledger_round_trip_and_reference_fields():
    """The ledger carries the reference's fields (a0, demean, scale, n_loop,
    n_scale, final_demean, mu) and packs back to the device record."""
    from steam_b200 import simulate as sim
    from steam_b200.ledger import BoundedAddLedger
    pert, mean, inc = _ba_case((40, 36, 16))
    led = sim._bounded_amplitude_add(pert.copy(), mean, inc.copy(), 0.0, 0.03)
    again = BoundedAddLedger.from_device(led.to_device(), led.n_rescale)
    for k in ('a0', 'demean', 'scale', 'n_loop', 'n_scale', 'final_demean', 'n_steps',
              'has_final'):
        np.testing.assert_array_equal(getattr(again, k), getattr(led, k), err_msg=k)
    np.testing.assert_array_equal(np.isnan(again.mu), np.isnan(led.mu))
    assert np.all(led.n_scale <= led.n_loop) and np.all(led.n_loop <= led.n_rescale)
    assert np.all(led.scale[:, :][led.n_steps[:, None] <= np.arange(led.n_rescale)] == 1.0)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_projection_replay_is_bit_exact(dtype):
    from steam_b200 import simulate as sim
    rng = np.random.default_rng(6)
    shape = (30, 20, 12)
    mean = np.linspace(0.001, 0.02, 12).astype(np.float32)
    pert = (0.004 * rng.standard_normal(shape)).astype(dtype)
    p_solve = pert.copy()
    led = sim._project_onto_bounds(p_solve, mean, 0.0, 0.03)
    assert np.any(led.violating) and not np.all(led.violating)
    p_rep = pert.copy()
    assert sim._project_onto_bounds(p_rep, mean, 0.0, 0.03, ledger=led) is led
    np.testing.assert_array_equal(p_rep, p_solve)


def test_simulate_replays_its_ledger_bit_for_bit():
    """A whole root run replayed from its own ledger: every class's flux
    advance, product norm and bounded add, and the composition's projection
    and flux restore, are injected instead of measured."""
    from steam_b200 import simulate as sim
    zp = np.arange(28) * 30.0
    args = dict(h_profile=340e3 - 20e3 * zp / zp.max(), qt_profile=0.018 - 0.016 * zp / zp.max(),
                nx=16, ny=16, dx=125.0, dy=125.0, outer_scale=2000.0, spheroscale=100.0,
                domain_height=800.0, profile_dz=30.0, output_path=None, seed=42)
    first = sim.simulate(**args)
    led = first['ledger']
    assert all(c.flux is not None and c.bounded_add for c in led.classes)
    again = sim.simulate(**args, ledger=led)
    for k in ('h', 'qt', 'flux'):
        np.testing.assert_array_equal(again[k], first[k], err_msg=k)


def test_replay_rejects_a_ledger_of_another_shape():
    from steam_b200 import simulate as sim
    pert, mean, inc = _ba_case((40, 36, 16))
    led = sim._bounded_amplitude_add(pert.copy(), mean, inc.copy(), 0.0, 0.03)
    p2, m2, i2 = _ba_case((40, 36, 12))
    with pytest.raises(ValueError):
        sim._bounded_amplitude_add(p2, m2, i2, 0.0, 0.03, ledger=led)
