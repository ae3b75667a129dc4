"""The out-of-core class step against the resident one (needs a B200).

streamed_class_step keeps the class's fields in host memory and streams
column tiles (plus their halo) and level slabs through the device
(steam/streaming.py:850-1447).  Every realized scalar is measured over the
whole class, so it reproduces the resident step up to the order of the
double-precision sums: the flux, the scalar increments and the condensate
agree to float32 rounding, integer counts exactly, and a repeat gives the
same bits.
"""

import numpy as np
import pytest

import config_cases as cc

pytestmark = pytest.mark.gpu


def _setup(shape, dtype):
    from steam_b200.ensemble import member_setup
    return member_setup(shape, seed=11, dtype=dtype)


def _inputs(shape, dtype, pinned):
    import torch
    h, q, F = cc.inputs(shape, seed=5)
    out = []
    for a in (h, q, F):
        a = a.astype(dtype)
        if pinned:
            t = torch.empty(shape, dtype=torch.float32 if dtype == np.float32 else torch.float64,
                            pin_memory=True)
            t.numpy()[...] = a
            a = t.numpy()
        out.append(a)
    return out


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape,tile,slab", [((96, 80, 64), (40, 36), 16),
                                             ((128, 128, 64), (128, 50), 24),
                                             ((64, 64, 32), (64, 64), 32)])
def test_streamed_class_step_matches_resident(dtype, shape, tile, slab):
    from steam_b200.outofcore import streamed_class_step
    from steam_b200.simulate import field_step
    setup = _setup(shape, dtype)
    h0, q0, F0 = _inputs(shape, dtype, pinned=False)
    h1, q1, F1 = h0.copy(), q0.copy(), F0.copy()
    d1, l1 = field_step(h1, q1, F1, setup)
    h2, q2, F2 = _inputs(shape, dtype, pinned=True)
    d2, l2 = streamed_class_step(h2, q2, F2, setup, tile=tile, slab_levels=slab)
    bar = 1e-6 if dtype == np.float32 else 1e-12
    assert rel(F2, F1) < bar
    assert rel(h2 - h0, h1 - h0) < 20 * bar
    assert rel(q2 - q0, q1 - q0) < 20 * bar
    for k in ('qc', 'qi'):
        assert rel(d2[k], d1[k]) < 20 * bar, k
    assert l2.flux.entering.count == l1.flux.entering.count
    assert l2.flux.noise_abs.count == l1.flux.noise_abs.count
    assert abs(l2.flux.n_clipped - l1.flux.n_clipped) <= 2
    for name in ('h', 'qt'):
        np.testing.assert_array_equal(l2.pattern[name].level_count,
                                      l1.pattern[name].level_count)
        assert rel(l2.pattern[name].level_total, l1.pattern[name].level_total) < bar
        assert rel(l2.bounded_add[name].a0, l1.bounded_add[name].a0) < bar


def test_streamed_class_step_repeats_bit_for_bit():
    from steam_b200.outofcore import streamed_class_step
    shape = (96, 80, 64)
    setup = _setup(shape, np.float32)
    runs = []
    for _ in range(2):
        h, q, F = _inputs(shape, np.float32, pinned=True)
        d, _ = streamed_class_step(h, q, F, setup, tile=(40, 36), slab_levels=16)
        runs.append((h.copy(), q.copy(), F.copy(), d['qc'].copy()))
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a, b)


def test_streamed_class_step_refuses_a_tile_whose_halo_wraps():
    from steam_b200.outofcore import streamed_class_step
    shape = (32, 32, 16)
    setup = _setup(shape, np.float32)
    h, q, F = _inputs(shape, np.float32, pinned=False)
    with pytest.raises(ValueError, match="halo"):
        streamed_class_step(h, q, F, setup, tile=(24, 32))
