"""The three-pass separable convolution (needs a B200).

Separable plans that the fused kernels do not take (the 41- and 61-tap
turbulons of sparsity 3.3 and 5, and any float64 field with such a kernel)
run as a z pass, a y pass and an x pass through HBM, each thread computing 8
consecutive outputs of its axis from a sliding register window.  Against the
FP64 oracle (steam/utils.py:293-427 semantics: x/y circular, z linear) on
interior-only shapes, partial tiles in every axis, periods shorter than the
kernel (several wraps in x and y), z thinner than the kernel, odd nz and
odd y-z planes, input and output at 4-byte offsets; with the input scaling
prologue, the flux epilogue on a window and the wide store; and at the
512 x 512 x 256 configuration's full size, float32 against the float64
device passes and linear in the input.

Bars: float64 1e-12 relative L2; float32 (float32 arithmetic in every pass)
1e-6 relative L2 (61 taps per pass, three roundings of intermediates).
"""

import ctypes

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib

pytestmark = pytest.mark.gpu

BAR = {np.float32: 1e-6, np.float64: 1e-12}
K61 = O.turbulon_envelope(1, 0.1, 0.1, 0.1, shape='mexican_hat', dtype=np.float64)
K41 = O.turbulon_envelope(1, 0.15, 0.15, 0.15, shape='mexican_hat', dtype=np.float64)
SHAPES = [(64, 64, 64), (72, 70, 52), (33, 22, 20), (16, 12, 8), (130, 40, 100), (24, 21, 13),
          (33, 21, 20)]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def U():
    from steam_b200 import utils
    return utils


def _launches(lib):
    return lib.steam_launch_count()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", SHAPES)
def test_three_passes_against_oracle(U, shape, dtype):
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape).astype(dtype)
    plan = U.plan_convolution(K61, shape, dtype)
    assert plan.kind == 'separable'
    ft = torch.as_tensor(f, device='cuda')
    out = torch.empty_like(ft)
    n0, p0 = _launches(lib), lib.steam_conv_packed_launches()
    U.run_plan(plan, ft, out)
    assert _launches(lib) - n0 == 3 and lib.steam_conv_packed_launches() == p0
    assert rel_l2(out.cpu().numpy(), O.convolve(f.astype(np.float64), K61)) < BAR[dtype]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_41_taps_against_oracle(U, dtype):
    import torch
    shape = (48, 50, 36)
    rng = np.random.default_rng(41)
    f = rng.standard_normal(shape).astype(dtype)
    plan = U.plan_convolution(K41, shape, dtype)
    assert plan.kind == 'separable'
    out = torch.empty(shape, dtype=torch.float32 if dtype == np.float32 else torch.float64,
                      device='cuda')
    U.run_plan(plan, torch.as_tensor(f, device='cuda'), out)
    assert rel_l2(out.cpu().numpy(), O.convolve(f.astype(np.float64), K41)) < BAR[dtype]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_prologue_against_oracle(U, dtype):
    import torch
    shape = (40, 70, 52)
    rng = np.random.default_rng(7)
    f = rng.standard_normal(shape).astype(dtype)
    div = (0.5 + rng.random(shape[2])).astype(dtype).astype(np.float64)
    mul = (0.5 + rng.random(shape[2])).astype(dtype).astype(np.float64)
    plan = U.plan_convolution(K61, shape, dtype)
    ft = torch.as_tensor(f, device='cuda')
    out = torch.empty_like(ft)
    U.run_plan(plan, ft, out, pre_div=div, pre_mul=mul)
    scale = (mul / div).astype(dtype).astype(np.float64)
    want = O.convolve(f.astype(np.float64) * scale[None, None, :], K61)
    assert rel_l2(out.cpu().numpy(), want) < BAR[dtype]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_flux_epilogue_on_a_window(U, dtype):
    """F = max(F + conv, 0) with the window sum and the clip count; float32
    fields take float64 arithmetic here, so the result is the float64 sum
    rounded once."""
    import torch
    shape = (36, 66, 56)
    rng = np.random.default_rng(9)
    f = (0.6 * rng.standard_normal(shape)).astype(dtype)
    F = (0.05 + 0.1 * rng.random(shape)).astype(dtype)
    window = (3, 31, 2, 60)
    plan = U.plan_convolution(K61, shape, dtype)
    new = F.astype(np.float64) + O.convolve(f.astype(np.float64), K61)
    want_clip = int(np.count_nonzero(new.astype(dtype) < 0))
    want = np.maximum(new, 0.0)
    assert want_clip > 0
    out = torch.as_tensor(F, device='cuda')
    sums = U.run_plan(plan, torch.as_tensor(f, device='cuda'), out,
                      epilogue=_lib.STEAM_EPI_FLUX, window=window)
    got = out.cpu().numpy()
    assert rel_l2(got, want) < (1e-12 if dtype == np.float64 else 5e-7)
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


def test_wide_store_against_oracle(U):
    """The wide store of a float32 field: float64 arithmetic in every pass,
    float32 intermediates and output."""
    import torch
    shape = (64, 48, 40)
    rng = np.random.default_rng(13)
    f = rng.standard_normal(shape).astype(np.float32)
    plan = U.plan_convolution(K61, shape, np.float32)
    ft = torch.as_tensor(f, device='cuda')
    a = torch.empty_like(ft)
    b = torch.empty_like(ft)
    U.run_plan(plan, ft, a)
    U.run_plan(plan, ft, b, epilogue=_lib.STEAM_EPI_STORE_WIDE)
    want = O.convolve(f.astype(np.float64), K61)
    assert rel_l2(b.cpu().numpy(), want) < 5e-7
    assert rel_l2(a.cpu().numpy(), want) < BAR[np.float32]


@pytest.mark.parametrize("in_offset,out_offset", [(1, 0), (0, 1), (1, 1)])
def test_unaligned_arrays(U, in_offset, out_offset):
    """Input and output at 4-byte offsets (no 8-byte pair access there)."""
    import torch
    shape = (40, 34, 26)
    n = shape[0] * shape[1] * shape[2]
    rng = np.random.default_rng(17)
    base_in = torch.as_tensor(rng.standard_normal(n + 1).astype(np.float32), device='cuda')
    f = base_in[in_offset:in_offset + n].view(shape)
    base_out = torch.zeros(n + 1, dtype=torch.float32, device='cuda')
    out = base_out[out_offset:out_offset + n].view(shape)
    plan = U.plan_convolution(K61, shape, np.float32)
    U.run_plan(plan, f, out)
    want = O.convolve(f.cpu().numpy().astype(np.float64), K61)
    assert rel_l2(out.cpu().numpy(), want) < BAR[np.float32]
    if out_offset:
        assert float(base_out[0]) == 0.0


def test_repeat_launches_are_bit_identical(U):
    import torch
    shape = (72, 70, 52)
    rng = np.random.default_rng(3)
    f = torch.as_tensor(rng.standard_normal(shape).astype(np.float32), device='cuda')
    plan = U.plan_convolution(K61, shape, np.float32)
    a, b = torch.empty_like(f), torch.empty_like(f)
    U.run_plan(plan, f, a)
    U.run_plan(plan, f, b)
    assert torch.equal(a, b)


def test_full_size_float32_against_float64_device():
    """The 512 x 512 x 256 configuration's 61^3 convolution: float32 passes
    (paired) against the float64 passes (scalar windows, held to 1e-12 of
    the FP64 oracle above) on the same field, and linear in its input."""
    import torch
    shape = (512, 512, 256)
    g = torch.Generator(device='cuda')
    g.manual_seed(61)
    f64 = torch.randn(shape, generator=g, device='cuda', dtype=torch.float64)
    f32 = f64.float()
    p32 = U_plan(shape, np.float32)
    p64 = U_plan(shape, np.float64)
    from steam_b200 import utils as U
    o32 = torch.empty_like(f32)
    o64 = torch.empty_like(f64)
    U.run_plan(p32, f32, o32)
    U.run_plan(p64, f32.double(), o64)
    rel = float(torch.linalg.vector_norm(o32.double() - o64) / torch.linalg.vector_norm(o64))
    assert rel < BAR[np.float32], rel
    # linearity: conv(2 f + h) = 2 conv(f) + conv(h)
    h32 = torch.randn(shape, generator=g, device='cuda', dtype=torch.float32)
    oh = torch.empty_like(h32)
    U.run_plan(p32, h32, oh)
    both = torch.empty_like(h32)
    U.run_plan(p32, 2.0 * f32 + h32, both)
    lin = (2.0 * o32.double() + oh.double())
    rel = float(torch.linalg.vector_norm(both.double() - lin) / torch.linalg.vector_norm(lin))
    assert rel < 2 * BAR[np.float32], rel


def U_plan(shape, dtype):
    from steam_b200 import utils as U
    plan = U.plan_convolution(K61, shape, dtype)
    assert plan.kind == 'separable'
    return plan
