"""The convolution for kernels without a separable form (needs a B200).

* The kernel spectrum built on the device against numpy's float64 FFT of the
  zero-padded kernel (the transform the reference takes with torch,
  steam/utils.py:367-375).
* The float32 overlap-save FFT convolution and the float64 direct sum against
  the FP64 oracle (steam/utils.py:293-427 semantics: x/y circular, z linear)
  on shapes that cut the 32^3 cubes unevenly, fields narrower than the kernel
  (the kernel longer than the period), fields thinner than the kernel in z,
  even kernel extents, one-tap axes and the 25-tap limit.
* The fused prologue (per-level input scaling) and the flux epilogue
  (F = max(F + conv, 0), window sum, clip count) against the same arithmetic
  in numpy, through both the synchronous and the device-scalar entry points.

Bars: float32 FFT against the float64 oracle 3e-6 relative L2 (a 32-point
transform's rounding, five stages per axis, forward and inverse); float64
direct sum 1e-12.
"""

import ctypes

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib

pytestmark = pytest.mark.gpu

FFT_BAR = 3e-6


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def brev5(i):
    return int(f"{i:05b}"[::-1], 2)


@pytest.fixture(scope="module")
def U():
    from steam_b200 import utils
    return utils


def _kernels():
    rng = np.random.default_rng(17)
    return {
        "morlet13": O.turbulon_envelope(1, 0.5, 0.5, 0.5, shape='morlet_omega0_6',
                                        dtype=np.float64),
        "rand537": rng.standard_normal((5, 7, 3)),
        "rand648": rng.standard_normal((6, 4, 8)),
        "rand13_1_13": rng.standard_normal((13, 1, 13)),
        "rand25": rng.standard_normal((25, 25, 25)),
    }


KERNELS = _kernels()


def test_spectrum_against_numpy_fft():
    import torch
    lib = _lib.load()
    for name, k in KERNELS.items():
        kx, ky, kz = k.shape
        kd = torch.as_tensor(k, device='cuda').contiguous()
        spec = torch.empty(lib.steam_conv_fft_spectrum_bytes(), dtype=torch.uint8, device='cuda')
        _lib.check(lib.steam_conv_fft_spectrum(_lib.ptr(kd), kx, ky, kz, _lib.ptr(spec),
                                               _lib.stream()))
        got = spec.view(torch.complex64).cpu().numpy().reshape(17, 32, 32)
        pad = np.zeros((32, 32, 32))
        pad[:kx, :ky, :kz] = k
        want = np.fft.rfftn(pad, axes=(0, 1, 2)) * (0.5 / 32 ** 3)  # [fx][fy][k]
        perm = [brev5(i) for i in range(32)]
        want = want.transpose(2, 0, 1)[:, perm][:, :, perm]
        assert rel_l2(got, want) < 1e-7, name


@pytest.mark.parametrize("shape", [(40, 36, 30), (7, 9, 20), (64, 48, 5), (33, 17, 70),
                                   (128, 128, 64), (20, 20, 20), (1, 1, 40)])
@pytest.mark.parametrize("kname", sorted(KERNELS))
def test_fft_convolution_against_oracle(U, shape, kname):
    k = KERNELS[kname]
    rng = np.random.default_rng(sum(shape) + len(kname))
    f = rng.standard_normal(shape).astype(np.float32)
    plan = U.plan_convolution(k, shape, np.float32)
    assert plan.kind == 'fft'
    got = U.convolve_fft_xy_oa_z(f, k)
    assert got.dtype == np.float32
    assert rel_l2(got, O.convolve(f.astype(np.float64), k)) < FFT_BAR


@pytest.mark.parametrize("shape", [(40, 36, 30), (7, 9, 20), (33, 17, 70)])
@pytest.mark.parametrize("kname", ["morlet13", "rand648"])
def test_direct_float64_against_oracle(U, shape, kname):
    k = KERNELS[kname]
    rng = np.random.default_rng(sum(shape))
    f = rng.standard_normal(shape)
    assert U.plan_convolution(k, shape, np.float64).kind == 'direct'
    got = U.convolve_fft_xy_oa_z(f, k)
    assert got.dtype == np.float64
    assert rel_l2(got, O.convolve(f, k)) < 1e-12


def test_direct_float32_kernel_longer_than_25_taps(U):
    rng = np.random.default_rng(2)
    k = rng.standard_normal((27, 5, 9))
    f = rng.standard_normal((40, 24, 30)).astype(np.float32)
    assert U.plan_convolution(k, f.shape, np.float32).kind == 'direct'
    got = U.convolve_fft_xy_oa_z(f, k)
    assert rel_l2(got, O.convolve(f.astype(np.float64), k)) < 1e-6


def _flux_reference(F, conv, window):
    new = F.astype(np.float64) + conv
    clipped = int(np.count_nonzero(new.astype(F.dtype) < 0))
    new = np.maximum(new.astype(F.dtype), 0)
    x0, x1, y0, y1 = window
    return new, float(new[x0:x1, y0:y1].astype(np.float64).sum()), clipped


@pytest.mark.parametrize("kind,dtype", [("fft", np.float32), ("direct", np.float64),
                                        ("direct", np.float32)])
def test_prologue_and_flux_epilogue(U, kind, dtype):
    import torch
    shape = (36, 30, 40)
    rng = np.random.default_rng(9)
    k = KERNELS["morlet13"]
    f = rng.standard_normal(shape).astype(dtype)
    F = (0.05 + 0.1 * rng.random(shape)).astype(dtype)
    div = (0.5 + rng.random(shape[2])).astype(dtype).astype(np.float64)
    mul = (0.5 + rng.random(shape[2])).astype(np.float32).astype(np.float64)
    window = (3, 31, 2, 27)
    plan = U.plan_convolution(k, shape, dtype)
    if kind == 'direct' and dtype == np.float32:
        plan = U.ConvPlan(kind='direct', shape=plan.shape, kernel=plan.kernel,
                          centre=plan.centre, device_data={})
    assert plan.kind == kind
    scale = (mul / div).astype(dtype)
    fs = (f * scale[None, None, :]).astype(dtype)
    conv = O.convolve(fs.astype(np.float64), k)
    want, want_sum, want_clip = _flux_reference(F, conv, window)
    assert want_clip > 0
    ft = torch.as_tensor(f, device='cuda')
    # synchronous entry: host prologue vectors, host sums
    out = torch.as_tensor(F, device='cuda')
    sums = U.run_plan(plan, ft, out, pre_div=div, pre_mul=mul, epilogue=_lib.STEAM_EPI_FLUX,
                      window=window)
    bar = FFT_BAR if kind == 'fft' else 1e-6 if dtype == np.float32 else 1e-12
    got = out.cpu().numpy()
    assert rel_l2(got, want) < bar
    assert sums[1] == (window[1] - window[0]) * (window[3] - window[2]) * shape[2]
    assert abs(sums[2] - want_clip) <= max(2, want_clip // 200)
    assert sums[0] == pytest.approx(want_sum, rel=10 * bar)
    # device-scalar entry: device prologue vector, device sums
    out2 = torch.as_tensor(F, device='cuda')
    pre = torch.as_tensor(np.concatenate([div, mul]).astype(dtype), device='cuda')
    sums_dev = torch.zeros(2, dtype=torch.float64, device='cuda')
    U.run_plan_async(plan, ft, out2, pre, _lib.STEAM_EPI_FLUX, window,
                     ctypes.c_void_p(sums_dev.data_ptr()))
    assert torch.equal(out, out2)
    s2 = sums_dev.cpu().numpy()
    assert s2[0] == sums[0] and s2[1] == sums[2]


def test_fft_store_async_equals_sync(U):
    import torch
    shape = (45, 38, 27)
    rng = np.random.default_rng(4)
    f = torch.as_tensor(rng.standard_normal(shape).astype(np.float32), device='cuda')
    plan = U.plan_convolution(KERNELS["morlet13"], shape, np.float32)
    a = torch.empty_like(f)
    b = torch.empty_like(f)
    U.run_plan(plan, f, a)
    U.run_plan_async(plan, f, b)
    assert torch.equal(a, b)
    # repeatable bit for bit
    c = torch.empty_like(f)
    U.run_plan_async(plan, f, c)
    assert torch.equal(b, c)


def test_fft_rejects_long_kernels():
    import torch
    lib = _lib.load()
    k = torch.zeros((26, 3, 3), dtype=torch.float64, device='cuda')
    spec = torch.empty(lib.steam_conv_fft_spectrum_bytes(), dtype=torch.uint8, device='cuda')
    rc = lib.steam_conv_fft_spectrum(_lib.ptr(k), 26, 3, 3, _lib.ptr(spec), _lib.stream())
    assert rc == 1
    assert b"25" in lib.steam_last_error()
