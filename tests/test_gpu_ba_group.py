"""Grouped bounded adds (needs a B200).

Several fields of different shapes, windows and bounds solved as one group
(``steam_bounded_add_group_*``: one launch per stage, per-field teams in the
persistent phases) against the oracle's bounded add of each field
(steam/simulate.py:3114-3283), against the single-field call and against
the same field solved alone (team sizes, hence block partials, depend on the
group); repeats of a group are bit-identical; the ledger records match the
single call's; and the grouped ensemble step agrees with the per-member one.

Bars: float32, a cell within twice the shift's stopping tolerance a0 2^-20
(the device stops once the root is bracketed that narrowly; the oracle's
bisection sits elsewhere inside the bracket) plus four roundings of the
largest bound (mu, d - mu, the clip and p + d each round once); float64,
1e-12 of the largest bound.
"""

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib

pytestmark = pytest.mark.gpu

N_RESCALE = 10


def _case(shape, seed, lo, hi):
    rng = np.random.default_rng(seed)
    nz = shape[2]
    span = hi - lo
    mean = np.linspace(lo + 0.02 * span, hi - 0.03 * span, nz)
    pert = np.clip(0.1 * span * rng.standard_normal(shape) + mean, lo, hi) - mean
    inc = 0.15 * span * rng.standard_normal(shape)
    inc[:, :, 3] = 0.0  # a clip-only level
    return pert, mean, inc


CASES = [((64, 48, 40), 1, 0.0, 0.03, None),
         ((40, 40, 16), 2, 315 * 1004.0, 355 * 1004.0, None),
         ((96, 64, 64), 3, 0.0, 0.03, (8, 88, 4, 60)),
         ((24, 32, 8), 4, -1.0, 1.0, None),
         ((128, 128, 32), 5, 0.0, 0.03, None)]


def _same_bits(a, b):
    """Bit-identical tensors (NaN entries of the ledger included)."""
    import torch
    if a.dtype == torch.float64:
        return torch.equal(a.view(torch.int64), b.view(torch.int64))
    return torch.equal(a.view(torch.int32), b.view(torch.int32))


def _f32_bar(a0, lo, hi):
    return 2 * np.ldexp(float(np.max(a0)), -20) + 4 * float(
        np.spacing(np.float32(max(abs(lo), abs(hi)))))


def _run_group(dtype, cases, torch):
    lib = _lib.load()
    code = _lib.STEAM_F32 if dtype == np.float32 else _lib.STEAM_F64
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    width = 7 + 2 * N_RESCALE
    fields, probs = [], []
    for shape, seed, lo, hi, win in cases:
        pert, mean, inc = _case(shape, seed, lo, hi)
        p = torch.as_tensor(pert.astype(dtype), device='cuda').contiguous()
        d = torch.as_tensor(inc.astype(dtype), device='cuda').contiguous()
        m = torch.as_tensor(mean.astype(dtype).astype(np.float64), device='cuda')
        led = torch.zeros(shape[2] * width, dtype=torch.float64, device='cuda')
        q = _lib.BAProblem()
        q.nx, q.ny, q.nz = shape
        q.pert, q.increment, q.mean = p.data_ptr(), d.data_ptr(), m.data_ptr()
        q.phi_min, q.phi_max = lo, hi
        q.has_window = 0 if win is None else 1
        if win is not None:
            q.window = _lib.Window(*win)
        q.ledger = led.data_ptr()
        probs.append(q)
        fields.append((p, d, m, led, pert, mean, inc))
    arr = (_lib.BAProblem * len(probs))(*probs)
    nbytes = lib.steam_bounded_add_group_workspace_bytes(code, len(probs), arr, N_RESCALE)
    ws = torch.empty(int(nbytes), dtype=torch.uint8, device='cuda')
    _lib.check(lib.steam_bounded_add_group_prepare(code, len(probs), arr, N_RESCALE,
                                                   _lib.ptr(ws), int(nbytes)))
    _lib.check(lib.steam_bounded_add_group_async(_lib.ptr(ws), _lib.stream()))
    torch.cuda.synchronize()
    return fields, ws, lib


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_group_against_oracle(dtype):
    import torch
    fields, ws, lib = _run_group(dtype, CASES, torch)
    try:
        for (shape, seed, lo, hi, win), (p, d, m, led, pert, mean, inc) in zip(CASES, fields):
            p_o = pert.astype(dtype)
            i_o = inc.astype(dtype)
            O.bounded_amplitude_add(p_o, mean.astype(dtype), i_o, lo, hi, window=win)
            got = p.cpu().numpy()
            a0 = led.cpu().numpy().reshape(shape[2], -1)[:, 0]
            assert np.all(led.cpu().numpy().reshape(shape[2], -1)[:, 4] > 0)  # sweeps run
            if dtype == np.float32:
                atol = _f32_bar(a0, lo, hi)
            else:
                atol = 1e-12 * max(abs(lo), abs(hi))
            np.testing.assert_allclose(got, p_o, rtol=0, atol=atol)
            field = got + mean.astype(dtype)[None, None, :]
            assert field.min() >= lo - atol and field.max() <= hi + atol
    finally:
        lib.steam_bounded_add_group_release(_lib.ptr(ws))


def test_group_matches_single_calls_and_alone():
    import torch
    from steam_b200 import simulate as sim
    dtype = np.float32
    fields, ws, lib = _run_group(dtype, CASES, torch)
    alone, ws1, _ = _run_group(dtype, CASES[2:3], torch)
    try:
        # field 2 alone and in the group (other team sizes, so other block
        # partials): the same solve to rounding
        a0 = alone[0][3].cpu().numpy().reshape(CASES[2][0][2], -1)[:, 0]
        np.testing.assert_allclose(alone[0][0].cpu().numpy(), fields[2][0].cpu().numpy(),
                                   rtol=0, atol=_f32_bar(a0, 0.0, 0.03))
        for (shape, seed, lo, hi, win), (p, d, m, led, pert, mean, inc) in zip(CASES, fields):
            p_s = pert.astype(dtype)
            rec = sim._bounded_amplitude_add(p_s, mean.astype(dtype), inc.astype(dtype), lo, hi,
                                             window=win)
            a0 = np.asarray(rec.a0)
            atol = _f32_bar(a0, lo, hi)
            np.testing.assert_allclose(p.cpu().numpy(), p_s, rtol=0, atol=atol)
            g = led.cpu().numpy().reshape(shape[2], -1)
            np.testing.assert_allclose(g[:, 0], a0, rtol=1e-6)
            assert np.array_equal(g[:, 1].astype(int), np.asarray(rec.n_loop))
    finally:
        lib.steam_bounded_add_group_release(_lib.ptr(ws))
        lib.steam_bounded_add_group_release(_lib.ptr(ws1))


def test_group_repeats_bit_for_bit():
    import torch
    fields, ws, lib = _run_group(np.float32, CASES, torch)
    try:
        first = [(f[0].clone(), f[3].clone()) for f in fields]
        for (p, d, m, led, pert, mean, inc) in fields:
            p.copy_(torch.as_tensor(pert.astype(np.float32)))
            d.copy_(torch.as_tensor(inc.astype(np.float32)))
        _lib.check(lib.steam_bounded_add_group_async(_lib.ptr(ws), _lib.stream()))
        torch.cuda.synchronize()
        for (a, la), f in zip(first, fields):
            assert _same_bits(a, f[0]) and _same_bits(la, f[3])
    finally:
        lib.steam_bounded_add_group_release(_lib.ptr(ws))


def test_group_rejects_unsupported_layouts():
    lib = _lib.load()
    q = _lib.BAProblem()
    q.nx, q.ny, q.nz = 8, 8, 6  # nz % 4 != 0
    q.pert = q.increment = q.mean = 256
    q.phi_min, q.phi_max = 0.0, 1.0
    arr = (_lib.BAProblem * 1)(q)
    assert lib.steam_bounded_add_group_prepare(_lib.STEAM_F32, 1, arr, N_RESCALE, 256, 1 << 20) != 0
    assert b"multiple of 4" in lib.steam_last_error()
    assert lib.steam_bounded_add_group_async(12345, None) != 0


def test_grouped_ensemble_step_against_per_member_step():
    import torch
    from steam_b200.ensemble import Ensemble, Member
    shapes = [(48, 48, 32), (64, 64, 48), (80, 80, 64), (32, 32, 32)]
    members = [Member(s, 1100 + j, alpha=1.6 + 0.1 * j) for j, s in enumerate(shapes)]
    ens = Ensemble(members, n_streams=2, tune=False, grouped=True)
    assert ens.grouped
    ens.step_eager()
    torch.cuda.synchronize()
    grouped = [(m.h.clone(), m.q.clone(), m.F.clone(), m.diag["qc"].clone()) for m in members]
    led_g = ens.check()
    ens.release()
    ens2 = Ensemble(members, n_streams=2, tune=False, grouped=False)
    assert not ens2.grouped
    ens2.step_eager()
    torch.cuda.synchronize()
    led_s = ens2.check()
    for m, g, lg, ls in zip(members, grouped, led_g, led_s):
        assert torch.equal(m.F, g[2])  # the flux advance is the same code
        for a, b in ((m.h, g[0]), (m.q, g[1])):
            rel = float(torch.linalg.vector_norm((a - b).double()) /
                        torch.linalg.vector_norm(b.double()))
            assert rel < 1e-6, rel
        for name in ('h', 'qt'):
            np.testing.assert_allclose(lg.bounded_add[name].a0, ls.bounded_add[name].a0,
                                       rtol=1e-6)
