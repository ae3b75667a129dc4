"""Full-size properties of the CUDA path (needs a B200).

At the workloads' full sizes -- the 2048x2048x256 FP32 field (1.07 G voxels)
and the 512x512x256 field in FP32 and FP64 -- the oracle is too slow to run,
so these tests check properties that hold at any size: the keyed integers
equal the oracle's at sampled sites of the whole world; world-keyed noise
restricts exactly (a box equals the same cells of the whole world, wrap
included, and sparse noise is nonzero on the centre lattice only); the
convolution commutes with periodic x/y shifts bit for bit and is linear to
rounding; the flux advance keeps the entering mean with F >= 0 and repeats
bit for bit; a class step keeps both scalars within their bounds, leaves
each level's applied increment at zero mean, splits total water exactly
into vapour and condensate, and repeats bit for bit.
"""

import numpy as np
import pytest

from oracle import steam_oracle as O

pytestmark = pytest.mark.gpu

WORLD = (2048, 2048, 256)


@pytest.fixture(autouse=True)
def _release():
    yield
    import torch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def _rel_l2(a, b):
    n = float(b.double().norm())
    return float((a.double() - b.double()).norm()) / (n if n > 0 else 1.0)


def test_keyed_integers_at_sampled_sites_of_the_full_world():
    import torch
    from steam_b200.noise import keyed_uniforms
    key = O.class_key(np.random.SeedSequence(2048))
    rng = np.random.default_rng(11)
    ix = np.concatenate([[0, 1, 2047], rng.integers(0, 2048, 21)])
    iy = np.concatenate([[0, 2046, 2047], rng.integers(0, 2048, 21)])
    iz = np.concatenate([[0, 255], rng.integers(0, 256, 22)])
    n = ix.size * iy.size * iz.size
    l0 = torch.empty(n, dtype=torch.float32, device='cuda')
    l1 = torch.empty(n, dtype=torch.float32, device='cuda')
    keyed_uniforms(torch.as_tensor(ix, device='cuda'), torch.as_tensor(iy, device='cuda'),
                   torch.as_tensor(iz, device='cuda'), *key, l0, l1)
    r0, r1 = O.keyed_uniforms(ix, iy, iz, key)
    assert np.array_equal(l0.cpu().numpy().view(np.uint32), r0.view(np.uint32))
    assert np.array_equal(l1.cpu().numpy().view(np.uint32), r1.view(np.uint32))


def test_world_noise_restricts_exactly_at_2048x2048x256():
    import torch
    from steam_b200 import simulate as sim
    key = O.class_key(np.random.SeedSequence(7))
    full = sim.levy_field_device(WORLD, (1, 1, 1), 1.8, sim.NoiseRegion(key, (0, 0, 0), WORLD))
    assert bool(torch.isfinite(full).all())
    for origin, shape in (((2040, 2030, 200), (16, 40, 56)), ((1000, 5, 0), (64, 33, 256)),
                          ((0, 2047, 17), (9, 3, 100))):
        box = sim.levy_field_device(shape, (1, 1, 1), 1.8, sim.NoiseRegion(key, origin, WORLD))
        xs = torch.as_tensor((origin[0] + np.arange(shape[0])) % WORLD[0], device='cuda')
        ys = torch.as_tensor((origin[1] + np.arange(shape[1])) % WORLD[1], device='cuda')
        cut = full.index_select(0, xs).index_select(1, ys)[:, :, origin[2]:origin[2] + shape[2]]
        assert torch.equal(box.view(torch.int32), cut.contiguous().view(torch.int32)), origin
    del full
    # sparse noise (centres every 5 cells): nonzero on the world lattice only
    # (a centre's draw is exactly 0 only when its phase uniform is exactly
    # 1/2, probability 2^-24 per centre, so a handful at most)
    sparse = sim.levy_field_device(WORLD, (5, 5, 5), 1.8, sim.NoiseRegion(key, (0, 0, 0), WORLD))
    on = [torch.arange(n, device='cuda') % 5 == 0 for n in WORLD]
    lattice = on[0][:, None, None] & on[1][None, :, None] & on[2][None, None, :]
    nonzero = sparse != 0
    assert not bool((nonzero & ~lattice).any())
    assert int((lattice & ~nonzero).sum()) <= 8


def test_convolution_commutes_with_periodic_shifts_at_2048x2048x256():
    import torch
    from steam_b200.utils import convolve_device
    kern = O.turbulon_envelope(1, 0.5, 0.5, 0.5)
    g = torch.Generator(device='cuda')
    g.manual_seed(5)
    f = torch.randn(WORLD, generator=g, device='cuda')
    out = convolve_device(f, kern)
    assert bool(torch.isfinite(out).all())
    shift = (37, 1029)
    f = torch.roll(f, shift, (0, 1))
    out_shifted = convolve_device(f, kern)
    del f
    # the same operations in the same order for every output cell, wherever
    # its tiles and x-chunks fall: equal bits
    assert torch.equal(out_shifted, torch.roll(out, shift, (0, 1)))


@pytest.mark.parametrize("dtype,tol", [("float32", 2e-6), ("float64", 1e-13)])
def test_convolution_is_linear_at_512x512x256(dtype, tol):
    import torch
    from steam_b200.utils import convolve_device
    tdt = getattr(torch, dtype)
    kern = O.turbulon_envelope(1, 0.5, 0.5, 0.5, dtype=np.dtype(dtype))
    g = torch.Generator(device='cuda')
    g.manual_seed(9)
    shape = (512, 512, 256)
    a = torch.randn(shape, generator=g, device='cuda', dtype=tdt)
    b = torch.rand(shape, generator=g, device='cuda', dtype=tdt)
    lhs = convolve_device(0.75 * a - 2.5 * b, kern)
    rhs = 0.75 * convolve_device(a, kern) - 2.5 * convolve_device(b, kern)
    assert _rel_l2(lhs, rhs) < tol


def test_flux_advance_keeps_the_mean_and_repeats_at_2048x2048x256():
    import torch
    from steam_b200 import simulate as sim
    from steam_b200.utils import plan_convolution
    kern = O.turbulon_envelope(1, 0.5, 0.5, 0.5)
    plan = plan_convolution(kern, WORLD, np.float32)
    region = sim.NoiseRegion(O.class_key(np.random.SeedSequence(21)), (0, 0, 0), WORLD)
    results = []
    for _ in range(2):
        F = torch.ones(WORLD, device='cuda')
        st = sim.advance_flux_device(F, region, plan, 0.1, 1, (1, 1, 1))
        del st
        results.append(F)
    F0, F1 = results
    assert torch.equal(F0, F1)
    assert float(F0.min()) >= 0.0
    # the restore returns the entering mean (1) up to the float32 rounding of
    # the factor and of each product
    mean = float(F0.double().mean())
    assert abs(mean - 1.0) < 1e-6
    assert float(F0.double().std()) > 1e-3  # the noise did move the flux


def _class_step(shape, dtype, seed):
    import torch
    from steam_b200.ensemble import Member
    m = Member(shape, seed, dtype=dtype)
    m.reset()
    m.step()
    torch.cuda.synchronize()
    return m


@pytest.mark.parametrize("shape,dtype", [(WORLD, np.float32), ((512, 512, 256), np.float64)])
def test_class_step_invariants_at_full_size(shape, dtype):
    import torch
    m = _class_step(shape, dtype, 1000)
    cs = m.setup
    h_min, h_max, q_min, q_max = cs.bounds
    tdt = m.h.dtype
    h_mean = torch.as_tensor(cs.h_mean, dtype=torch.float64, device='cuda')
    q_mean = torch.as_tensor(cs.qt_mean, dtype=torch.float64, device='cuda')
    eps = 2e-6 if dtype == np.float32 else 1e-12
    # the bounded add keeps the composed scalars within their bounds (level
    # extremes of the perturbation plus the level mean)
    for pert, mean, lo, hi in ((m.h, h_mean, h_min, h_max), (m.q, q_mean, q_min, q_max)):
        span = hi - lo
        assert float((pert.amin(dim=(0, 1)).double() + mean).min()) >= lo - eps * span
        assert float((pert.amax(dim=(0, 1)).double() + mean).max()) <= hi + eps * span
    # each level's applied increment has zero mean (the solved shift): to the
    # solver's bracket, far below the level's mean amplitude
    ncol = shape[0] * shape[1]
    for pert, pert0, name in ((m.h, m.h0, 'h'), (m.q, m.q0, 'qt')):
        inc = pert - pert0
        lvl_mean = inc.sum(dim=(0, 1), dtype=torch.float64) / ncol
        lvl_amp = inc.abs().sum(dim=(0, 1), dtype=torch.float64) / ncol
        del inc
        ok = lvl_amp > 0
        assert bool(ok.any()), name
        rel = (lvl_mean[ok].abs() / lvl_amp[ok]).max()
        assert float(rel) < (1e-4 if dtype == np.float32 else 1e-9), name
    # the flux kept its entering mean and stayed non-negative
    assert float(m.F.min()) >= 0.0
    m_in = float(m.F0.sum(dtype=torch.float64)) / m.F0.numel()
    m_out = float(m.F.sum(dtype=torch.float64)) / m.F.numel()
    assert abs(m_out - m_in) < (2e-6 if dtype == np.float32 else 1e-12) * m_in
    # thermodynamics: total water splits into vapour and condensate, the
    # condensate is non-negative, the pressure falls with height
    d = m.diag
    qt = (m.q + q_mean.to(tdt)).clamp(q_min, q_max)
    water = d['qv'] + d['qc'] + d['qi']
    tol_w = 8 * float(torch.finfo(tdt).eps) * float(qt.abs().max())
    assert float((water - qt).abs().max()) <= tol_w
    del water, qt
    assert float(d['qc'].min()) >= 0.0 and float(d['qi'].min()) >= 0.0
    assert bool((d['p'][:, :, 1:] < d['p'][:, :, :-1]).all())
    assert bool(torch.isfinite(d['T']).all())
    # a second step from the same state: the same bits
    sums = [float(t.sum(dtype=torch.float64)) for t in (m.h, m.q, m.F, d['qc'], d['qi'])]
    keep = [t.clone() for t in (m.h, m.q, m.F, d['qc'], d['qi'])]
    m.reset()
    m.step()
    torch.cuda.synchronize()
    for a, b in zip(keep, (m.h, m.q, m.F, d['qc'], d['qi'])):
        assert torch.equal(a, b)
    assert sums == [float(t.sum(dtype=torch.float64)) for t in (m.h, m.q, m.F, d['qc'], d['qi'])]
