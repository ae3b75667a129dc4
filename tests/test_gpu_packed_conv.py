"""The packed float32 fused convolution (needs a B200).

The separable 13-tap turbulon filters on float32 fields run on the packed
kernel (tensor-copied slabs, f32x2 arithmetic): against the FP64 oracle
(steam/utils.py:293-427 semantics: x/y circular, z linear) on shapes with
interior tiles only, rows that wrap (edge tiles), fields narrower in y than a
tile's staged rows or thinner in z than its staged columns, partial y and z
tiles and x chunks that wrap; with the
input scaling prologue and the flux epilogue; against the scalar fused kernel
with float64 accumulation; bit for bit across x chunks; and with no slab wait
given up.

Bars: float32 against the float64 oracle 5e-7 relative L2 (the scalar fused
float32 kernel sits at ~1.5e-7, the reference's float32 FFT at ~2.2e-7).
"""

import ctypes

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib

pytestmark = pytest.mark.gpu

BAR = 5e-7
K64 = O.turbulon_envelope(1, 0.5, 0.5, 0.5, shape='mexican_hat', dtype=np.float64)
SHAPES = [(64, 64, 64), (40, 70, 52), (20, 40, 48), (33, 96, 96), (128, 128, 64),
          (16, 30, 16), (14, 22, 8)]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def U():
    from steam_b200 import utils
    return utils


def _wait_errors(lib):
    n = ctypes.c_int32(-1)
    _lib.check(lib.steam_take_wait_errors(ctypes.byref(n)))
    return n.value


def _packed_ran(lib, before):
    return lib.steam_conv_packed_launches() > before


@pytest.mark.parametrize("shape", SHAPES)
def test_packed_store_against_oracle(U, shape):
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape).astype(np.float32)
    plan = U.plan_convolution(K64, shape, np.float32)
    assert plan.kind == 'separable'
    ft = torch.as_tensor(f, device='cuda')
    out = torch.empty_like(ft)
    n0 = lib.steam_conv_packed_launches()
    U.run_plan(plan, ft, out)
    assert _packed_ran(lib, n0)
    assert rel_l2(out.cpu().numpy(), O.convolve(f.astype(np.float64), K64)) < BAR
    assert _wait_errors(lib) == 0


@pytest.mark.parametrize("shape", [(40, 70, 52), (64, 64, 64)])
def test_packed_prologue_against_oracle(U, shape):
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(7)
    f = rng.standard_normal(shape).astype(np.float32)
    div = (0.5 + rng.random(shape[2])).astype(np.float32).astype(np.float64)
    mul = (0.5 + rng.random(shape[2])).astype(np.float32).astype(np.float64)
    plan = U.plan_convolution(K64, shape, np.float32)
    out = torch.empty(shape, dtype=torch.float32, device='cuda')
    n0 = lib.steam_conv_packed_launches()
    U.run_plan(plan, torch.as_tensor(f, device='cuda'), out, pre_div=div, pre_mul=mul)
    assert _packed_ran(lib, n0)
    scale = (mul / div).astype(np.float32).astype(np.float64)
    want = O.convolve(f.astype(np.float64) * scale[None, None, :], K64)
    assert rel_l2(out.cpu().numpy(), want) < BAR


def test_packed_flux_epilogue(U):
    import torch
    lib = _lib.load()
    shape = (36, 66, 56)
    rng = np.random.default_rng(9)
    f = (0.6 * rng.standard_normal(shape)).astype(np.float32)
    F = (0.05 + 0.1 * rng.random(shape)).astype(np.float32)
    window = (3, 31, 2, 60)
    plan = U.plan_convolution(K64, shape, np.float32)
    conv = O.convolve(f.astype(np.float64), K64)
    new = F.astype(np.float64) + conv
    want_clip = int(np.count_nonzero(new.astype(np.float32) < 0))
    want = np.maximum(new, 0.0)
    assert want_clip > 0
    out = torch.as_tensor(F, device='cuda')
    n0 = lib.steam_conv_packed_launches()
    sums = U.run_plan(plan, torch.as_tensor(f, device='cuda'), out,
                      epilogue=_lib.STEAM_EPI_FLUX, window=window)
    assert _packed_ran(lib, n0)
    got = out.cpu().numpy()
    assert rel_l2(got, want) < BAR
    x0, x1, y0, y1 = window
    assert sums[0] == pytest.approx(float(got[x0:x1, y0:y1].astype(np.float64).sum()),
                                    rel=1e-12)
    assert sums[1] == (x1 - x0) * (y1 - y0) * shape[2]
    assert abs(sums[2] - want_clip) <= max(2, want_clip // 200)
    # the device-scalar entry gives the same bits
    out2 = torch.as_tensor(F, device='cuda')
    sums_dev = torch.zeros(2, dtype=torch.float64, device='cuda')
    U.run_plan_async(plan, torch.as_tensor(f, device='cuda'), out2, None,
                     _lib.STEAM_EPI_FLUX, window, ctypes.c_void_p(sums_dev.data_ptr()))
    assert torch.equal(out, out2)
    s2 = sums_dev.cpu().numpy()
    assert s2[0] == sums[0] and s2[1] == sums[2]


def test_packed_against_float64_accumulation(U):
    """The same flux advance on the packed float32 kernel and on the scalar
    fused kernel with float64 taps and accumulators, on dense noise (every
    cell a centre, so the convolution is O(1) and many cells sit near the
    clip): within the log-flux bar of each other."""
    import torch
    lib = _lib.load()
    shape = (64, 64, 64)
    rng = np.random.default_rng(3)
    f = torch.as_tensor((0.3 * rng.standard_normal(shape)).astype(np.float32), device='cuda')
    F = torch.as_tensor((1.0 + 0.1 * rng.random(shape)).astype(np.float32), device='cuda')
    plan = U.plan_convolution(K64, shape, np.float32)
    a = F.clone()
    U.run_plan(plan, f, a, epilogue=_lib.STEAM_EPI_FLUX)
    try:
        _lib.check(lib.steam_conv_set_flux_wide(1))
        n0 = lib.steam_conv_packed_launches()
        b = F.clone()
        U.run_plan(plan, f, b, epilogue=_lib.STEAM_EPI_FLUX)
        assert lib.steam_conv_packed_launches() == n0
    finally:
        _lib.check(lib.steam_conv_set_flux_wide(0))
    clear = (a > 1e-3) & (b > 1e-3)
    assert int(((a > 0) != (b > 0)).sum()) <= 2
    la, lb = torch.log(a[clear].double()), torch.log(b[clear].double())
    assert float(torch.linalg.vector_norm(la - lb) / torch.linalg.vector_norm(lb)) < 1e-5


def test_packed_unaligned_input_takes_the_scalar_kernel(U):
    import torch
    lib = _lib.load()
    shape = (24, 40, 48)
    rng = np.random.default_rng(5)
    base = torch.as_tensor(rng.standard_normal(24 * 40 * 48 + 1).astype(np.float32),
                           device='cuda')
    f = base[1:].view(shape)  # 4-byte offset: no tensor copy from here
    out = torch.empty(shape, dtype=torch.float32, device='cuda')
    plan = U.plan_convolution(K64, shape, np.float32)
    n0 = lib.steam_conv_packed_launches()
    U.run_plan(plan, f, out)
    assert lib.steam_conv_packed_launches() == n0
    want = O.convolve(f.cpu().numpy().astype(np.float64), K64)
    assert rel_l2(out.cpu().numpy(), want) < BAR


def test_packed_chunks_are_bit_identical(U):
    import torch
    lib = _lib.load()
    shape = (96, 64, 64)
    rng = np.random.default_rng(11)
    f = torch.as_tensor(rng.standard_normal(shape).astype(np.float32), device='cuda')
    plan = U.plan_convolution(K64, shape, np.float32)
    outs = []
    try:
        for chunk in (0, 16, 48, 96, 256):
            _lib.check(lib.steam_conv_set_xchunk(*shape, chunk))
            o = torch.empty_like(f)
            U.run_plan(plan, f, o)
            outs.append(o)
    finally:
        _lib.check(lib.steam_conv_set_xchunk(*shape, 0))
    for o in outs[1:]:
        assert torch.equal(o, outs[0])
    assert _wait_errors(lib) == 0


@pytest.mark.parametrize("shape", [(40, 70, 52), (33, 96, 96), (24, 130, 64)])
def test_packed_tile_heights_are_bit_identical(U, shape):
    """The 64-row tile (512 threads) against the 32-row tile: the same bits,
    and the oracle's result; the autotuner's setting is per shape."""
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(len(shape) + shape[1])
    f = torch.as_tensor(rng.standard_normal(shape).astype(np.float32), device='cuda')
    F = torch.as_tensor((1.0 + 0.1 * rng.random(shape)).astype(np.float32), device='cuda')
    plan = U.plan_convolution(K64, shape, np.float32)
    outs, fluxes = [], []
    try:
        for rows in (32, 64):
            _lib.check(lib.steam_conv_set_tile_rows(*shape, rows))
            assert lib.steam_conv_get_tile_rows(*shape) == rows
            o = torch.empty_like(f)
            U.run_plan(plan, f, o)
            outs.append(o)
            fl = F.clone()
            U.run_plan(plan, 0.3 * f, fl, epilogue=_lib.STEAM_EPI_FLUX)
            fluxes.append(fl)
    finally:
        _lib.check(lib.steam_conv_set_tile_rows(*shape, 0))
    assert lib.steam_conv_get_tile_rows(*shape) == 32
    assert torch.equal(outs[0], outs[1])
    assert torch.equal(fluxes[0], fluxes[1])
    want = O.convolve(f.cpu().numpy().astype(np.float64), K64)
    assert rel_l2(outs[1].cpu().numpy(), want) < BAR
    assert lib.steam_conv_set_tile_rows(*shape, 48) != 0
    assert _wait_errors(lib) == 0
